// extern "C" entry points of libamber_cuda (declared in include/amber_cuda.h)
// and the host-side control flow that replaces the rp loop of 4_fbe/amber.c /
// amber_v2.c: grid upload + normalisation, ring geometry, calCR, closed-form
// triplet counts, and per-r1-group map building followed by the per-triangle
// contraction.
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <set>
#include <map>
#include <vector>

#include "lagspace.cuh"

namespace amber {

int fail(amber_cuda_ctx *c, int code, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

int cuda_check(amber_cuda_ctx *c, cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return AMBER_OK;
    return fail(c, e == cudaErrorMemoryAllocation ? AMBER_ERR_OOM : AMBER_ERR_CUDA, "%s: %s", what,
                cudaGetErrorString(e));
}

int ensure(amber_cuda_ctx *c, DevBuf &b, size_t bytes, const char *what)
{
    if (bytes <= b.bytes) return AMBER_OK;
    size_t want = std::max(bytes, b.bytes + b.bytes / 4);
    if (c->held - b.bytes + want > c->budget) {
        want = bytes;
        if (c->held - b.bytes + want > c->budget)
            return fail(c, AMBER_ERR_OOM, "%s: %zu bytes would exceed the HBM budget (%zu held of %zu)", what, bytes,
                        c->held, c->budget);
    }
    if (b.p) {
        cudaStreamSynchronize(c->stream);
        cudaFree(b.p);
        c->held -= b.bytes;
        b.p = nullptr;
        b.bytes = 0;
    }
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(c, AMBER_ERR_OOM, "%s: cudaMalloc(%zu) failed: %s", what, want, cudaGetErrorString(e));
    }
    b.bytes = want;
    c->held += want;
    return AMBER_OK;
}

static void release(amber_cuda_ctx *c, DevBuf &b)
{
    if (b.p) {
        cudaFree(b.p);
        c->held -= b.bytes;
    }
    b.p = nullptr;
    b.bytes = 0;
}

int twiddle_table(amber_cuda_ctx *c, long n, const double2 **out)
{
    auto it = c->twiddles.find(n);
    if (it == c->twiddles.end()) {
        std::vector<double2> h(n);
        for (long k = 0; k <= n / 2; ++k) {
            long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)n;
            h[k] = make_double2((double)cosl(a), (double)sinl(a));
        }
        // exactly conjugate-symmetric, e^{2πi(n−k)/n} = conj(e^{2πik/n}): the map builder
        // evaluates pixels x and n − x from one twiddle
        for (long k = n / 2 + 1; k < n; ++k) h[k] = make_double2(h[n - k].x, -h[n - k].y);
        DevBuf b;
        int rc = ensure(c, b, sizeof(double2) * n, "twiddle table");
        if (rc) return rc;
        rc = cuda_check(c, cudaMemcpy(b.p, h.data(), sizeof(double2) * n, cudaMemcpyHostToDevice), "twiddles");
        if (rc) return rc;
        it = c->twiddles.emplace(n, b).first;
    }
    *out = reinterpret_cast<const double2 *>(it->second.p);
    return AMBER_OK;
}

void phase_begin(amber_cuda_ctx *c, int phase)
{
    if (c->phase_used == c->phase_ev.size()) {
        amber_cuda_ctx::PhaseEv e;
        cudaEventCreate(&e.a);
        cudaEventCreate(&e.b);
        c->phase_ev.push_back(e);
    }
    c->phase_ev[c->phase_used].phase = phase;
    cudaEventRecord(c->phase_ev[c->phase_used].a, c->stream);
}

void phase_end(amber_cuda_ctx *c)
{
    cudaEventRecord(c->phase_ev[c->phase_used].b, c->stream);
    ++c->phase_used;
}

namespace {

// normalize_data (amber_funcs.c:1946-1978): GV /= NTiG where NTiG > 0, then
// NTiG := 1 there (it becomes the 0/1 sampling mask).
__global__ void normalize_kernel(const double2 *__restrict__ sums, const double *__restrict__ counts, long n,
                                 double2 *__restrict__ grid, double *__restrict__ mask)
{
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double2 v = sums[i];
        double t = counts[i];
        if (t > 0) {
            v.x /= t;
            v.y /= t;
            t = 1;
        }
        grid[i] = v;
        mask[i] = t;
    }
}

long ng1_of(double uhigh, double du)
{
    // amber.c:193-197
    double umax = uhigh + 3;
    long nmax = (long)(umax / du);
    long ng = (long)(3 * nmax);
    return (ng % 2 == 0) ? ng + 2 : ng + 3;
}

bool closed(const std::vector<double> &ua, int r1, int r2, int r3)
{
    // calCR's rule, amber_funcs.c:439-449
    double tt = ua[r2] / ua[r1];
    if (!(tt >= 0.5 && tt <= 1.0)) return false;
    double mu = 0.5 * (tt + 1. / tt - (ua[r3] / ua[r1]) * (ua[r3] / ua[r2]));
    return mu >= 0.5 / tt && mu <= 1.0;
}

int check_ready(amber_cuda_ctx *c, bool need_channels)
{
    if (!c->grid.p) return fail(c, AMBER_ERR_STATE, "no grid loaded");
    if (c->Nr <= 0) return fail(c, AMBER_ERR_STATE, "no rings set");
    for (int r = 0; r < c->Nr; ++r)
        if (c->uhigh[r] > c->N1 / 2)
            return fail(c, AMBER_ERR_ARG, "ring %d reaches U=%g beyond the grid half-width %ld", r, c->uhigh[r],
                        c->N1 / 2);
    if (need_channels && c->nc10 < 0) return fail(c, AMBER_ERR_STATE, "no channels set");
    if (need_channels && (long)c->weight.size() != c->nc)
        return fail(c, AMBER_ERR_STATE, "channels were set for a different channel count");
    return AMBER_OK;
}

int upload_grid(amber_cuda_ctx *c, long N1, long nc, double Du, int flag_key, const double *re_im,
                const double *ntig, bool on_device = false)
{
    if (N1 <= 0 || N1 % 2 || nc <= 0 || !(Du > 0) || !re_im || !ntig)
        return fail(c, AMBER_ERR_ARG, "bad grid arguments (N1=%ld nc=%ld Du=%g)", N1, nc, Du);
    if (flag_key != 0 && flag_key != 1) return fail(c, AMBER_ERR_ARG, "flag_key must be 0 or 1 (got %d)", flag_key);
    const long n = N1 * (N1 / 2 + 1) * nc;
    int rc;
    if ((rc = ensure(c, c->grid, sizeof(double2) * n, "grid"))) return rc;
    if ((rc = ensure(c, c->mask, sizeof(double) * n, "sampling mask"))) return rc;
    const double2 *raw;
    const double *cnt;
    if (on_device) {
        // normalised straight from the caller's device buffers
        raw = (const double2 *)re_im;
        cnt = ntig;
    } else {
        // the raw sums land in the partial buffer first, then normalise into grid/mask
        if ((rc = ensure(c, c->partial, sizeof(double2) * n + sizeof(double) * n, "grid staging"))) return rc;
        double2 *sraw = (double2 *)c->partial.p;
        double *scnt = (double *)((char *)c->partial.p + sizeof(double2) * n);
        if ((rc = cuda_check(c, cudaMemcpyAsync(sraw, re_im, sizeof(double2) * n, cudaMemcpyHostToDevice, c->stream),
                             "upload grid")))
            return rc;
        if ((rc = cuda_check(c, cudaMemcpyAsync(scnt, ntig, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream),
                             "upload sampling")))
            return rc;
        raw = sraw;
        cnt = scnt;
    }
    normalize_kernel<<<4 * c->num_sms, 256, 0, c->stream>>>(raw, cnt, n, (double2 *)c->grid.p, (double *)c->mask.p);
    if ((rc = cuda_check(c, cudaGetLastError(), "normalize launch"))) return rc;
    c->N1 = N1;
    c->nc = nc;
    c->Du = Du;
    c->flag_key = flag_key;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "grid upload");
}

}  // namespace

long ring_ng1(double uhigh, double du) { return ng1_of(uhigh, du); }

std::vector<int> closed_triangles(const std::vector<double> &ulow, const std::vector<double> &uhigh)
{
    const int Nr = (int)ulow.size();
    std::vector<double> ua(Nr);
    for (int i = 0; i < Nr; ++i)  // amber_funcs.c:2065, as amber_cuda_set_rings
        ua[i] = (2. / 3.) * (pow(uhigh[i], 3.) - pow(ulow[i], 3.)) / (pow(uhigh[i], 2.) - pow(ulow[i], 2.));
    std::vector<int> tri;
    for (int r1 = 0; r1 < Nr; ++r1)
        for (int r2 = 0; r2 <= r1; ++r2)
            for (int r3 = 0; r3 <= r2; ++r3)
                if (closed(ua, r1, r2, r3)) {
                    tri.push_back(r1);
                    tri.push_back(r2);
                    tri.push_back(r3);
                }
    return tri;
}

// ---- one realisation's triangles, run in map-set batches ----

int run_begin(amber_cuda_ctx *c, RunState &st, int ntri, const int *tri, int want_v2)
{
    if (!c || ntri < 0 || (ntri > 0 && !tri)) return AMBER_ERR_ARG;
    int rc = check_ready(c, true);
    if (rc) return rc;
    for (int t = 0; t < ntri; ++t) {
        int r1 = tri[3 * t], r2 = tri[3 * t + 1], r3 = tri[3 * t + 2];
        if (r1 < 0 || r1 >= c->Nr || r2 < 0 || r2 >= c->Nr || r3 < 0 || r3 >= c->Nr)
            return fail(c, AMBER_ERR_ARG, "triangle %d has a ring outside [0, %d)", t, c->Nr);
    }
    cudaSetDevice(c->device);
    const int nclen = 2 * c->nc10 + 1;
    const long ncsize = (long)nclen * nclen;
    if ((rc = ensure(c, c->results, sizeof(double) * 2 * ncsize * std::max(1, ntri), "results"))) return rc;
    st = RunState();
    st.tri.assign(tri, tri + 3 * ntri);
    st.want_v2 = want_v2;
    // group by r1: every ring of a group lives on the group's Ng1 grid
    for (int t = 0; t < ntri; ++t) {
        int r1 = tri[3 * t];
        long ng = ng1_of(c->uhigh[r1], c->Du);
        auto it = std::find_if(st.groups.begin(), st.groups.end(), [&](const RunState::Group &g) { return g.r1 == r1; });
        if (it == st.groups.end()) {
            st.groups.push_back(RunState::Group{r1, ng, {}});
            it = st.groups.end() - 1;
        }
        it->tris.push_back(t);
    }
    return AMBER_OK;
}

size_t map_slot_bytes(int precision, long ng, long nc, int want_v2)
{
    const size_t vbytes = precision == AMBER_PREC_FP64 ? 8 : (precision == AMBER_PREC_MIXED ? 7 : 4);
    const long kalign = precision == AMBER_PREC_MIXED ? LS_BLOCK : 64;
    const long k = ng * ng, kp = (k + kalign - 1) / kalign * kalign;
    const size_t per_pass = vbytes * (size_t)nc * kp + 8 * (size_t)nc + 4 * (size_t)(kp / LS_BLOCK + 1);
    // + the map builder's column-pass intermediate (double2 per ring row, column and channel)
    const size_t y = sizeof(double2) * (size_t)ng * (size_t)(ng / 3 + 1) * (size_t)nc;
    return per_pass * (want_v2 ? 2 : 1) + y;
}

int run_next_batch(amber_cuda_ctx *c, RunState &st, std::vector<I8Job> *jobs)
{
    int rc;
    while (st.gi < st.groups.size() && st.ti >= st.groups[st.gi].tris.size()) {
        ++st.gi;
        st.ti = 0;
    }
    if (st.gi >= st.groups.size()) return 0;
    const RunState::Group &g = st.groups[st.gi];
    const int *tri = st.tri.data();
    const int want_v2 = st.want_v2;
    const int prec = c->precision;
    const int nclen = 2 * c->nc10 + 1;
    const long ncsize = (long)nclen * nclen;
    double *res = (double *)c->results.p;
    const size_t vbytes = prec == AMBER_PREC_FP64 ? 8 : (prec == AMBER_PREC_MIXED ? 7 : 4);
    const long kalign = prec == AMBER_PREC_MIXED ? LS_BLOCK : 64;
    const long k = g.ng * g.ng, kp = (k + kalign - 1) / kalign * kalign;
    const long nblk = kp / LS_BLOCK;
    const size_t per_slot = vbytes * (size_t)c->nc * kp + 8 * (size_t)c->nc + 4 * (size_t)(nblk + 1);
    // The next batch of the group: triangles whose ring union fits the budget.
    size_t spare = c->budget > c->held ? c->budget - c->held : 0;
    spare += c->maps_d.bytes + c->maps_i.bytes + c->y.bytes;
    // keep room for the mixed-precision contraction's partial tiles when they live in this context
    const size_t reserve = ((size_t)64 << 20) +
                           (prec == AMBER_PREC_MIXED && !c->contracts_elsewhere ? contract_partial_cap(c) : 0);
    const long cap_slots = (long)((spare > reserve ? spare - reserve : 0) /
                                  (map_slot_bytes(prec, g.ng, c->nc, want_v2) + 1));
    if (cap_slots < 3) return fail(c, AMBER_ERR_OOM, "maps of one triangle (Ng1=%ld) exceed the budget", g.ng);
    std::vector<int> batch;
    std::set<int> rings;
    while (st.ti < g.tris.size()) {
        int t = g.tris[st.ti];
        std::set<int> u = rings;
        u.insert(tri[3 * t]);
        u.insert(tri[3 * t + 1]);
        u.insert(tri[3 * t + 2]);
        if ((long)u.size() > cap_slots) break;
        rings = u;
        batch.push_back(t);
        ++st.ti;
    }
    MapSet ms;
    ms.ng = g.ng;
    ms.k = k;
    ms.kp = kp;
    for (int i = 0; i < 256; ++i) ms.slot_of_ring[i] = -1;
    for (int r : rings) {
        ms.slot_of_ring[r] = (int)ms.ring_of_slot.size();
        ms.ring_of_slot.push_back(r);
    }
    ms.nslots = (int)ms.ring_of_slot.size();
    const size_t nvals = (size_t)ms.nslots * c->nc * kp;
    if ((rc = ensure(c, c->maps_d, per_slot * ms.nslots, "ring maps"))) return rc;
    if (want_v2 && (rc = ensure(c, c->maps_i, per_slot * ms.nslots, "ring mask maps"))) return rc;
    // carve one map set (D or I) out of its buffer
    auto carve = [&](void *base, MapJob &job, DigitMaps *dm_base) {
        char *p = (char *)base;
        if (prec == AMBER_PREC_FP64) {
            job.out_f64 = (double *)p;
        } else if (prec == AMBER_PREC_BF16X3) {
            job.out_hi = (uint16_t *)p;
            job.out_lo = (uint16_t *)p + nvals;
        } else {
            job.out_f32 = (float *)p;
            job.weight = (const int *)c->d_weight.p;
            job.dig = (int8_t *)(p + 4 * nvals);
            job.bexp = (int *)(p + 7 * nvals);
            if (dm_base) {
                dm_base->f32 = job.out_f32;
                dm_base->dig = job.dig;
                dm_base->bexp = job.bexp;
            }
        }
    };
    std::vector<I8Job> local;
    std::vector<I8Job> *jl = jobs ? jobs : &local;
    std::vector<F64Job> f64jobs;
    DigitMaps dmaps[2];
    for (int pass = 0; pass < (want_v2 ? 2 : 1); ++pass) {
        MapJob job{};
        job.src = pass == 0 ? c->grid.p : c->mask.p;
        job.src_complex = pass == 0;
        job.n1 = c->N1;
        job.nc = c->nc;
        job.chan_base = 0;
        job.nch = c->nc;
        job.ng = g.ng;
        job.kp = kp;
        job.nslots = ms.nslots;
        for (int r : ms.ring_of_slot) {
            job.lo.push_back(c->ulow[r]);
            job.hi.push_back(c->uhigh[r]);
        }
        carve(pass == 0 ? c->maps_d.p : c->maps_i.p, job, &dmaps[pass]);
        phase_begin(c, 0);
        rc = build_maps(c, job);
        phase_end(c);
        if (rc) return rc;
    }
    for (int t : batch) {
        const size_t s1 = ms.slot_of_ring[tri[3 * t]], s2 = ms.slot_of_ring[tri[3 * t + 1]],
                     s3 = ms.slot_of_ring[tri[3 * t + 2]];
        const size_t ss = (size_t)c->nc * kp;
        for (int pass = 0; pass < (want_v2 ? 2 : 1); ++pass) {
            void *base = pass == 0 ? c->maps_d.p : c->maps_i.p;
            double *lag = res + ((size_t)t * 2 + pass) * ncsize;
            if (prec == AMBER_PREC_MIXED) {
                const DigitMaps &b = dmaps[pass];
                auto slot = [&](size_t s) {
                    DigitMaps d;
                    d.f32 = b.f32 + s * ss;
                    d.dig = b.dig + s * 3 * ss;
                    d.bexp = b.bexp + s * nblk;
                    return d;
                };
                I8Job jb;
                jb.m1 = slot(s1); jb.m2 = slot(s2); jb.m3 = slot(s3);
                jb.k = k; jb.kp = kp;
                jb.nc = (int)c->nc; jb.nc10 = c->nc10;
                jb.weight = &c->weight;
                jb.nanchors = (int)c->anchors.size();
                jb.mask_pass = pass == 1;
                jb.lag_out = lag;
                jl->push_back(jb);
                rc = AMBER_OK;
            } else if (prec == AMBER_PREC_BF16X3) {
                const uint16_t *hi = (const uint16_t *)base;
                const uint16_t *lo = hi + nvals;
                rc = contract_bf16x3(c, hi + s1 * ss, lo + s1 * ss, hi + s2 * ss, lo + s2 * ss, hi + s3 * ss,
                                     lo + s3 * ss, k, kp, lag);
            } else {
                const double *m = (const double *)base;
                f64jobs.push_back(F64Job{m + s1 * ss, m + s2 * ss, m + s3 * ss, k, kp, lag});
            }
            if (rc) return rc;
        }
        c->last_products += (double)c->total_vcp * (double)k * (want_v2 ? 2.0 : 1.0);
    }
    if (!local.empty() && (rc = contract_i8_jobs(c, local))) return rc;
    if (!f64jobs.empty() && (rc = contract_fp64_jobs(c, f64jobs))) return rc;
    return 1;
}

}  // namespace amber


using namespace amber;

extern "C" {

void amber_cuda_default_opts(amber_cuda_opts *o)
{
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->precision = AMBER_PREC_MIXED;
}

int amber_cuda_create(const amber_cuda_opts *opts, amber_cuda_ctx **out)
{
    if (!out) return AMBER_ERR_ARG;
    *out = nullptr;
    amber_cuda_opts o;
    amber_cuda_default_opts(&o);
    if (opts) o = *opts;
    if (o.precision != AMBER_PREC_FP64 && o.precision != AMBER_PREC_MIXED && o.precision != AMBER_PREC_BF16X3 &&
        o.precision != AMBER_PREC_FP64_ABS)
        return AMBER_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= o.device) {
        cudaGetLastError();
        return AMBER_ERR_NODEV;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, o.device) != cudaSuccess || prop.major != 10) return AMBER_ERR_NODEV;
    if (cudaSetDevice(o.device) != cudaSuccess) return AMBER_ERR_NODEV;
    amber_cuda_ctx *c = new amber_cuda_ctx();
    c->device = o.device;
    c->precision = o.precision == AMBER_PREC_FP64_ABS ? AMBER_PREC_FP64 : o.precision;
    c->fp64_abs = o.precision == AMBER_PREC_FP64_ABS;
    c->chunk_px = o.chunk_px;
    if (o.tile_n != 0 && o.tile_n != 32 && o.tile_n != 64 && o.tile_n != 128) {
        delete c;
        return AMBER_ERR_ARG;
    }
    c->tile_n = o.tile_n;
    c->num_sms = prop.multiProcessorCount;
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    c->budget = o.hbm_budget ? o.hbm_budget : (size_t)(0.9 * (double)fr);
    if (o.stream) {
        c->stream = (cudaStream_t)o.stream;
    } else {
        cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        c->own_stream = true;
    }
    cudaEventCreate(&c->ev0);
    cudaEventCreate(&c->ev1);
    cudaEventCreate(&c->tev0);
    cudaEventCreate(&c->tev1);
    *out = c;
    return AMBER_OK;
}

void amber_cuda_destroy(amber_cuda_ctx *c)
{
    if (!c) return;
    amber::engine_shutdown(c);
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    DevBuf *bufs[] = {&c->grid, &c->mask, &c->d_weight, &c->d_anchors, &c->y, &c->maps_d, &c->maps_i,
                      &c->partial, &c->results, &c->ring_lohi, &c->misc, &c->mixed_scratch, &c->lagred, &c->jobdesc, &c->lagtrial, &c->lsred};
    for (DevBuf *b : bufs) release(c, *b);
    if (c->stage) cudaFreeHost(c->stage);
    c->stage = nullptr;
    for (auto &kv : c->twiddles) release(c, kv.second);
    for (auto &e : c->phase_ev) {
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->tev0) cudaEventDestroy(c->tev0);
    if (c->tev1) cudaEventDestroy(c->tev1);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char *amber_cuda_last_error(const amber_cuda_ctx *c)
{
    return c ? c->err.c_str() : "no context";
}

int amber_cuda_load_grid_packed(amber_cuda_ctx *c, long N1, long nc, double Du, int flag_key, const double *re_im,
                                const double *ntig)
{
    if (!c) return AMBER_ERR_ARG;
    cudaSetDevice(c->device);
    return upload_grid(c, N1, nc, Du, flag_key, re_im, ntig);
}

int amber_cuda_load_grid_device(amber_cuda_ctx *c, long N1, long nc, double Du, int flag_key, const double *re_im,
                                const double *ntig)
{
    if (!c) return AMBER_ERR_ARG;
    cudaSetDevice(c->device);
    cudaPointerAttributes a{}, b{};
    if (re_im && ntig &&
        (cudaPointerGetAttributes(&a, re_im) != cudaSuccess || cudaPointerGetAttributes(&b, ntig) != cudaSuccess ||
         a.type != cudaMemoryTypeDevice || b.type != cudaMemoryTypeDevice || a.device != c->device ||
         b.device != c->device)) {
        cudaGetLastError();
        return fail(c, AMBER_ERR_ARG, "load_grid_device: re_im and ntig must be device memory of device %d", c->device);
    }
    return upload_grid(c, N1, nc, Du, flag_key, re_im, ntig, true);
}

int amber_cuda_load_grid(amber_cuda_ctx *c, long N1, long nc, double Du, int flag_key, const double *const *GVre,
                         const double *const *GVim, const double *const *NTiG)
{
    if (!c) return AMBER_ERR_ARG;
    if (!GVre || !GVim || !NTiG || N1 <= 0 || nc <= 0) return fail(c, AMBER_ERR_ARG, "bad grid arguments");
    const long ncell = N1 * (N1 / 2 + 1);
    std::vector<double> ri((size_t)ncell * nc * 2), nt((size_t)ncell * nc);
    for (long i = 0; i < ncell; ++i) {
        if (!GVre[i] || !GVim[i] || !NTiG[i]) return fail(c, AMBER_ERR_ARG, "NULL cell pointer at %ld", i);
        for (long ch = 0; ch < nc; ++ch) {
            ri[(i * nc + ch) * 2] = GVre[i][ch];
            ri[(i * nc + ch) * 2 + 1] = GVim[i][ch];
            nt[i * nc + ch] = NTiG[i][ch];
        }
    }
    cudaSetDevice(c->device);
    return upload_grid(c, N1, nc, Du, flag_key, ri.data(), nt.data());
}

int amber_cuda_set_rings(amber_cuda_ctx *c, int Nr, const double *ULow, const double *UHigh)
{
    if (!c) return AMBER_ERR_ARG;
    if (Nr <= 0 || Nr > 255 || !ULow || !UHigh) return fail(c, AMBER_ERR_ARG, "bad ring count %d", Nr);
    for (int r = 0; r < Nr; ++r)
        if (!(UHigh[r] > ULow[r]) || !(ULow[r] >= 0))
            return fail(c, AMBER_ERR_ARG, "ring %d has edges [%g, %g)", r, ULow[r], UHigh[r]);
    c->Nr = Nr;
    c->ulow.assign(ULow, ULow + Nr);
    c->uhigh.assign(UHigh, UHigh + Nr);
    c->uavg.resize(Nr);
    for (int i = 0; i < Nr; ++i)  // amber_funcs.c:2065
        c->uavg[i] =
            (2. / 3.) * (pow(UHigh[i], 3.) - pow(ULow[i], 3.)) / (pow(UHigh[i], 2.) - pow(ULow[i], 2.));
    return AMBER_OK;
}

int amber_cuda_get_uavg(const amber_cuda_ctx *c, double *Uavg)
{
    if (!c || !Uavg || c->Nr <= 0) return AMBER_ERR_ARG;
    memcpy(Uavg, c->uavg.data(), sizeof(double) * c->Nr);
    return AMBER_OK;
}

int amber_cuda_set_channels(amber_cuda_ctx *c, int nc10, int uf_nc, const int *uf_chans)
{
    if (!c) return AMBER_ERR_ARG;
    if (c->nc <= 0) return fail(c, AMBER_ERR_STATE, "load the grid before the channels");
    if (nc10 < 0 || nc10 >= c->nc) return fail(c, AMBER_ERR_ARG, "nc10=%d outside [0, nc)", nc10);
    if (uf_nc < 0 || (uf_nc > 0 && !uf_chans)) return fail(c, AMBER_ERR_ARG, "bad uf_chans");
    std::vector<int> w(c->nc, uf_nc > 0 ? 0 : 1);
    for (int i = 0; i < uf_nc; ++i) {
        if (uf_chans[i] < 0 || uf_chans[i] >= c->nc)
            return fail(c, AMBER_ERR_ARG, "uf_chans[%d]=%d outside [0, %ld)", i, uf_chans[i], c->nc);
        w[uf_chans[i]] += 1;
    }
    const int nclen = 2 * nc10 + 1;
    // numdnu[Δ2][Δ3] = Σ_p1 w[p1]·w[p1+Δ2]·w[p1+Δ3]: the number of rows of the
    // reference's vcp table with that lag (amber_funcs.c:2207-2310), exactly.
    std::vector<int64_t> cnt((size_t)nclen * nclen, 0);
    std::vector<int> anchors;
    for (int p1 = 0; p1 < c->nc; ++p1) {
        if (!w[p1]) continue;
        anchors.push_back(p1);
        for (int d2 = -nc10; d2 <= nc10; ++d2) {
            int p2 = p1 + d2;
            if (p2 < 0 || p2 >= c->nc || !w[p2]) continue;
            int64_t w12 = (int64_t)w[p1] * w[p2];
            int64_t *row = cnt.data() + (size_t)(d2 + nc10) * nclen;
            for (int d3 = -nc10; d3 <= nc10; ++d3) {
                int p3 = p1 + d3;
                if (p3 < 0 || p3 >= c->nc || !w[p3]) continue;
                row[d3 + nc10] += w12 * w[p3];
            }
        }
    }
    int rc;
    if ((rc = ensure(c, c->d_weight, sizeof(int) * c->nc, "channel weights"))) return rc;
    if ((rc = ensure(c, c->d_anchors, sizeof(int) * std::max<size_t>(1, anchors.size()), "anchors"))) return rc;
    cudaSetDevice(c->device);
    if ((rc = cuda_check(c, cudaMemcpy(c->d_weight.p, w.data(), sizeof(int) * c->nc, cudaMemcpyHostToDevice),
                         "weights")))
        return rc;
    if (!anchors.empty() &&
        (rc = cuda_check(c, cudaMemcpy(c->d_anchors.p, anchors.data(), sizeof(int) * anchors.size(),
                                       cudaMemcpyHostToDevice),
                         "anchors")))
        return rc;
    c->nc10 = nc10;
    c->last_ntri = 0;  // the results buffer is laid out for the previous lag width
    c->uf.assign(uf_chans, uf_chans + uf_nc);
    c->weight = w;
    c->anchors = anchors;
    c->counts = cnt;
    c->total_vcp = 0;
    for (int64_t v : cnt) c->total_vcp += v;
    return AMBER_OK;
}

long amber_cuda_ng1(const amber_cuda_ctx *c, int r1)
{
    if (!c || r1 < 0 || r1 >= c->Nr || !(c->Du > 0)) return -1;
    return ng1_of(c->uhigh[r1], c->Du);
}

int amber_cuda_calcr(amber_cuda_ctx *c, int max_tri, int *rcount, double *rdata)
{
    if (!c || !rcount || (max_tri > 0 && !rdata)) return AMBER_ERR_ARG;
    int rc = check_ready(c, false);
    if (rc) return rc;
    const int plane = 5;  // calCR reads the channel-5 mask, amber_funcs.c:427
    if (c->nc <= plane) return fail(c, AMBER_ERR_ARG, "calCR reads channel %d but nc=%ld", plane, c->nc);
    cudaSetDevice(c->device);
    const long n1 = c->N1, k = n1 * n1;
    if ((rc = ensure(c, c->maps_i, sizeof(double) * (size_t)c->Nr * k, "calCR mask maps"))) return rc;
    MapJob job{};
    job.src = c->mask.p;
    job.src_complex = false;
    job.n1 = n1;
    job.nc = c->nc;
    job.chan_base = plane;
    job.nch = 1;
    job.ng = n1;
    job.kp = k;
    job.nslots = c->Nr;
    job.lo = c->ulow;
    job.hi = c->uhigh;
    job.out_f64 = (double *)c->maps_i.p;
    if ((rc = build_maps(c, job))) return rc;
    std::vector<int> tri;
    for (int r1 = 0; r1 < c->Nr; ++r1)
        for (int r2 = 0; r2 <= r1; ++r2)
            for (int r3 = 0; r3 <= r2; ++r3)
                if (closed(c->uavg, r1, r2, r3)) {
                    tri.push_back(r1);
                    tri.push_back(r2);
                    tri.push_back(r3);
                }
    const int n = (int)tri.size() / 3;
    if ((rc = ensure(c, c->results, sizeof(double) * std::max(1, n), "calCR sums"))) return rc;
    c->last_ntri = 0;  // the sums below overwrite the last triangle run's lag arrays
    if ((rc = triple_sums(c, (const double *)c->maps_i.p, k, tri, (double *)c->results.p))) return rc;
    std::vector<double> num(std::max(1, n));
    if ((rc = cuda_check(c, cudaMemcpyAsync(num.data(), c->results.p, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                            c->stream),
                         "calCR download")))
        return rc;
    if ((rc = cuda_check(c, cudaStreamSynchronize(c->stream), "calCR"))) return rc;
    *rcount = n;
    for (int t = 0; t < n && t < max_tri; ++t) {
        rdata[4 * t] = tri[3 * t];
        rdata[4 * t + 1] = tri[3 * t + 1];
        rdata[4 * t + 2] = tri[3 * t + 2];
        rdata[4 * t + 3] = num[t];
    }
    return AMBER_OK;
}

int amber_cuda_triangles_run(amber_cuda_ctx *c, int ntri, const int *tri, int want_v2)
{
    amber::RunState st;
    int rc = amber::run_begin(c, st, ntri, tri, want_v2);
    if (rc) return rc;
    c->last_products = 0;
    c->phase_used = 0;
    c->launches = 0;
    c->contractions = 0;
    cudaEventRecord(c->ev0, c->stream);
    const bool mixed = c->precision == AMBER_PREC_MIXED;
    std::vector<amber::I8Job> jobs;
    while ((rc = amber::run_next_batch(c, st, mixed ? &jobs : nullptr)) == 1) {
        // mixed path: the whole batch (every triangle and pass) in persistent launches
        if (mixed && (rc = amber::contract_i8_jobs(c, jobs))) return rc;
        jobs.clear();
    }
    if (rc < 0) return rc;
    cudaEventRecord(c->ev1, c->stream);
    if ((rc = cuda_check(c, cudaEventSynchronize(c->ev1), "triangle run"))) return rc;
    if ((rc = cuda_check(c, cudaGetLastError(), "triangle run"))) return rc;
    cudaEventElapsedTime(&c->last_ms, c->ev0, c->ev1);
    for (int i = 0; i < 3; ++i) c->phase_ms[i] = 0;
    for (size_t i = 0; i < c->phase_used; ++i) {
        float ms = 0;
        cudaEventElapsedTime(&ms, c->phase_ev[i].a, c->phase_ev[i].b);
        c->phase_ms[c->phase_ev[i].phase] += ms;
    }
    c->last_ntri = ntri;
    c->last_v2 = want_v2;
    return AMBER_OK;
}

int amber_cuda_triangles_fetch(amber_cuda_ctx *c, double *bldnu, int64_t *numdnu, double *numtri)
{
    if (!c) return AMBER_ERR_ARG;
    const int nclen = 2 * c->nc10 + 1;
    const long ncsize = (long)nclen * nclen;
    const int n = c->last_ntri;
    int rc;
    cudaSetDevice(c->device);
    for (int t = 0; t < n; ++t) {
        const double *src = (const double *)c->results.p + (size_t)t * 2 * ncsize;
        if (bldnu &&
            (rc = cuda_check(c, cudaMemcpyAsync(bldnu + (size_t)t * ncsize, src, sizeof(double) * ncsize,
                                                cudaMemcpyDeviceToHost, c->stream),
                             "fetch bldnu")))
            return rc;
        if (numtri && c->last_v2 &&
            (rc = cuda_check(c, cudaMemcpyAsync(numtri + (size_t)t * ncsize, src + ncsize, sizeof(double) * ncsize,
                                                cudaMemcpyDeviceToHost, c->stream),
                             "fetch numtri")))
            return rc;
        if (numdnu) memcpy(numdnu + (size_t)t * ncsize, c->counts.data(), sizeof(int64_t) * ncsize);
    }
    return cuda_check(c, cudaStreamSynchronize(c->stream), "fetch");
}

int amber_cuda_triangles(amber_cuda_ctx *c, int ntri, const int *tri, int want_v2, double *bldnu, int64_t *numdnu,
                         double *numtri)
{
    int rc = amber_cuda_triangles_run(c, ntri, tri, want_v2);
    if (rc) return rc;
    return amber_cuda_triangles_fetch(c, bldnu, numdnu, numtri);
}

int amber_cuda_shard_plan(int ntri, const int *r1, const long *ng1, int world, int *rank_of)
{
    if (ntri < 0 || world < 1 || (ntri > 0 && (!r1 || !ng1 || !rank_of))) return AMBER_ERR_ARG;
    // r1 groups in ascending r1, each holding its triangles in ascending index
    std::map<int, std::vector<int>> groups;
    std::map<int, long long> cost1;
    for (int t = 0; t < ntri; ++t) {
        if (ng1[t] <= 0) return AMBER_ERR_ARG;
        groups[r1[t]].push_back(t);
        cost1[r1[t]] = (long long)ng1[t] * ng1[t];
    }
    long long total = 0;
    for (const auto &g : groups) total += (long long)g.second.size() * cost1[g.first];
    struct Part {
        long long cost, map_cost;
        int r1;
        std::vector<int> tri;
    };
    std::vector<Part> parts;
    for (const auto &g : groups) {
        const long long n = (long long)g.second.size(), gcost = n * cost1[g.first];
        const long long m = std::max(1LL, std::min(n, (gcost * world + total - 1) / std::max(total, 1LL)));
        for (long long j = 0; j < m; ++j) {
            Part p;
            p.r1 = g.first;
            for (long long i = j; i < n; i += m) p.tri.push_back(g.second[(size_t)i]);
            p.cost = (long long)p.tri.size() * cost1[g.first];
            p.map_cost = gcost;  // in units of 1/25: the group's map building
            parts.push_back(std::move(p));
        }
    }
    std::stable_sort(parts.begin(), parts.end(), [](const Part &a, const Part &b) {
        if (a.cost != b.cost) return a.cost > b.cost;
        if (a.r1 != b.r1) return a.r1 < b.r1;
        return a.tri[0] < b.tri[0];
    });
    std::vector<long long> load(world, 0);  // 25 × cost + map costs
    for (const Part &p : parts) {
        int k = 0;
        for (int i = 1; i < world; ++i)
            if (load[i] < load[k]) k = i;
        for (int t : p.tri) rank_of[t] = k;
        load[k] += 25 * p.cost + p.map_cost;
    }
    return AMBER_OK;
}

int amber_cuda_tile_choices(const amber_cuda_ctx *c, int max_entries, int *nclen_class, int *tile_n,
                            float *ms_trial_32, float *ms_trial_64)
{
    if (!c || max_entries < 0) return AMBER_ERR_ARG;
    int n = 0;
    for (const auto &kv : c->tile_tuned) {
        if (n < max_entries) {
            if (nclen_class) nclen_class[n] = kv.first;
            if (tile_n) tile_n[n] = kv.second;
            for (const auto &t : c->tile_trials) {
                if (t.first == kv.first * 100 + 32 && ms_trial_32) ms_trial_32[n] = t.second;
                if (t.first == kv.first * 100 + 64 && ms_trial_64) ms_trial_64[n] = t.second;
            }
        }
        ++n;
    }
    return n;
}

int amber_cuda_last_run_stats(const amber_cuda_ctx *c, double *products, double *device_ms)
{
    if (!c) return AMBER_ERR_ARG;
    if (products) *products = c->last_products;
    if (device_ms) *device_ms = c->last_ms;
    return AMBER_OK;
}

int amber_cuda_last_run_breakdown(const amber_cuda_ctx *c, double *ms_maps, double *ms_contract, double *ms_reduce,
                                  long *kernel_launches, long *contract_launches)
{
    if (!c) return AMBER_ERR_ARG;
    if (ms_maps) *ms_maps = c->phase_ms[0];
    if (ms_contract) *ms_contract = c->phase_ms[1];
    if (ms_reduce) *ms_reduce = c->phase_ms[2];
    if (kernel_launches) *kernel_launches = c->launches;
    if (contract_launches) *contract_launches = c->contractions;
    return AMBER_OK;
}

int amber_cuda_last_run_shape(const amber_cuda_ctx *c, int *ntri, int *nclen, int *v2)
{
    if (!c) return AMBER_ERR_ARG;
    if (ntri) *ntri = c->last_ntri;
    if (nclen) *nclen = 2 * c->nc10 + 1;
    if (v2) *v2 = c->last_v2;
    return AMBER_OK;
}

int amber_cuda_triangle_v1(amber_cuda_ctx *c, int r1, int r2, int r3, double rdata_num, float *bldnu,
                           int32_t *numdnu, double *Ntri, double *Num)
{
    if (!c || !bldnu || !numdnu) return AMBER_ERR_ARG;
    int tri[3] = {r1, r2, r3};
    int rc = amber_cuda_triangles_run(c, 1, tri, 0);
    if (rc) return rc;
    const int nclen = 2 * c->nc10 + 1;
    const long ncsize = (long)nclen * nclen;
    std::vector<double> bl(ncsize);
    if ((rc = amber_cuda_triangles_fetch(c, bl.data(), nullptr, nullptr))) return rc;
    for (long i = 0; i < ncsize; ++i) {
        if (c->counts[i] > INT32_MAX)
            return fail(c, AMBER_ERR_OVERFLOW, "lag cell %ld holds %lld triplets, beyond int32", i,
                        (long long)c->counts[i]);
        bldnu[i] = (float)bl[i];
        numdnu[i] = (int32_t)c->counts[i];
    }
    // per-triangle scalars, amber.c:193-202,287
    long ng = ng1_of(c->uhigh[r1], c->Du);
    double gfact = (1. * ng) / (1. * c->N1);
    double num = gfact * gfact * rdata_num;
    double inv = 1.0 / (ng * ng * 1.);
    if (Num) *Num = num;
    if (Ntri) *Ntri = num * inv;
    return AMBER_OK;
}

int amber_cuda_triangle_v2(amber_cuda_ctx *c, int r1, int r2, int r3, float *bldnu, float *numdnu,
                           double *inv_Ng1_Ng2)
{
    if (!c || !bldnu || !numdnu) return AMBER_ERR_ARG;
    int tri[3] = {r1, r2, r3};
    int rc = amber_cuda_triangles_run(c, 1, tri, 1);
    if (rc) return rc;
    const int nclen = 2 * c->nc10 + 1;
    const long ncsize = (long)nclen * nclen;
    std::vector<double> bl(ncsize), nt(ncsize);
    if ((rc = amber_cuda_triangles_fetch(c, bl.data(), nullptr, nt.data()))) return rc;
    for (long i = 0; i < ncsize; ++i) {
        bldnu[i] = (float)bl[i];
        numdnu[i] = (float)nt[i];
    }
    long ng = ng1_of(c->uhigh[r1], c->Du);
    if (inv_Ng1_Ng2) *inv_Ng1_Ng2 = 1.0 / (ng * ng * 1.);
    return AMBER_OK;
}

}  // extern "C"
