// Cylindrical bispectrum from the lag arrays, on the device: the analysis
// stage's lag→k step (mabs_funcs.py get_cyl_BS 376-389 with fold_quadrants
// 210-222, cut_nan 259-260 and Bdnu2Bk_fft 325-334; the windowed form of
// mfunc_winds.py mabs_win 88-103 and cylbs_win 122-136 with blackman_nuttall
// 17-31), for every triangle of the last run at once.
//
// For one triangle, with L the lag array [Δ2][Δ3] (nclen = 2·nc10 + 1 rows and
// columns), C its normaliser (the triplet counts, or the sampling-mask sums of
// a v2 run) and n the edge cut:
//   fold:    F[r][c] = L[nc10][c]                               r = 0
//            F[r][c] = L[nc10 + r][c] + L[nc10 − r][nclen−1−c]   r = 1 .. nc10
//   ratio:   T = F(L / s_t) / mabs_norm / F(C)   (s_t: the caller's per-triangle divisor,
//            Num for the v1 chain, whose reader returns bldnu / Num; 1 when none is given)
//   cut:     D[m][k] = T[m][n + k]      m < M = nc10 + 1 − n,  k < N = nclen − 2n
//   window:  D[m][k] ·= w[N/2 + m] · w[k]   (Blackman–Nuttall of length N), optional
//   k-space: out = fftshift(irfft2(ifftshift(D, axis 1), axes (1, 0), s = (N, N)))
//            · rc⁴ · (N · dν · rc′)²
// irfft2 over axes (1, 0): a complex inverse DFT along axis 1, then a real
// inverse along axis 0 whose input is the half spectrum (M = N/2 + 1 rows, N
// odd), both with numpy's 1/N normalisation, ignoring Im of row 0.
//
// The transforms are direct FP64 sums (N ≤ 367 for the largest cube here), one
// thread per output value over a twiddle table in shared memory.
#include <math.h>

#include <algorithm>
#include <vector>

#include "common.cuh"

namespace amber {

namespace {

constexpr int kT = 256;

// fold + ratio + cut + window + ifftshift along the columns: d[t][m][k]
__global__ void cylbs_fold(const double *__restrict__ num, long num_stride, const double *__restrict__ den,
                           long den_stride, const double *__restrict__ tri_inv, int nc10, int ncut, double inv_norm,
                           const double *__restrict__ win, double *__restrict__ d)
{
    const int nclen = 2 * nc10 + 1;
    const int M = nc10 + 1 - ncut, N = nclen - 2 * ncut;
    const int t = blockIdx.y;
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long)M * N) return;
    const int m = (int)(e / N), kk = (int)(e % N);
    // ifftshift: output column kk holds input column (kk + N/2) mod N
    const int k = (kk + N / 2) % N;
    const int c = ncut + k;
    const double *L = num + (long)t * num_stride;
    const double *C = den + (long)t * den_stride;
    auto fold = [&](const double *a) {
        double v = a[(long)(nc10 + m) * nclen + c];
        if (m > 0) v += a[(long)(nc10 - m) * nclen + (nclen - 1 - c)];
        return v;
    };
    const double a = tri_inv ? fold(L) * tri_inv[t] : fold(L);
    double v = a * inv_norm / fold(C);
    if (win) v *= win[N / 2 + m] * win[k];
    d[((long)t * M + m) * N + kk] = v;
}

// X[t][m][x] = Σ_k d[t][m][k] e^{+2πi k x/N}
__global__ void cylbs_rows(const double *__restrict__ d, int M, int N, const double2 *__restrict__ tw_g,
                           double2 *__restrict__ X)
{
    extern __shared__ double2 tw[];
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = tw_g[i];
    __syncthreads();
    const int t = blockIdx.z, m = blockIdx.y;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= N) return;
    const double *row = d + ((long)t * M + m) * N;
    double re = 0.0, im = 0.0;
    int idx = 0;
    for (int k = 0; k < N; ++k) {
        const double v = row[k];
        re = fma(v, tw[idx].x, re);
        im = fma(v, tw[idx].y, im);
        idx += x;
        if (idx >= N) idx -= N;
    }
    X[((long)t * M + m) * N + x] = make_double2(re, im);
}

// out[t][(y+N/2)%N][(x+N/2)%N] = scale/N² · (Re X[0][x] + 2 Σ_{m≥1} Re(X[m][x] e^{+2πi m y/N}))
__global__ void cylbs_cols(const double2 *__restrict__ X, int M, int N, const double2 *__restrict__ tw_g,
                           double scale, double *__restrict__ out)
{
    extern __shared__ double2 tw[];
    for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = tw_g[i];
    __syncthreads();
    const int t = blockIdx.z, y = blockIdx.y;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= N) return;
    const double2 *Xt = X + (long)t * M * N;
    double acc = 0.0;
    int idx = y;  // twiddle index m·y mod N, starting at m = 1
    for (int m = 1; m < M; ++m) {
        const double2 v = Xt[(long)m * N + x];
        acc = fma(v.x, tw[idx].x, acc);
        acc = fma(-v.y, tw[idx].y, acc);
        idx += y;
        if (idx >= N) idx -= N;
    }
    const double r = (Xt[x].x + 2.0 * acc) * scale / ((double)N * (double)N);
    const int ys = (y + N / 2) % N, xs = (x + N / 2) % N;
    out[((long)t * N + ys) * N + xs] = r;
}

}  // namespace

// Device bytes amber_cuda_cyl_bs may add to a context: its scratch (normalisers, window,
// one batch of d / X / out) and the twiddle table.
size_t cyl_bs_bytes(int nc10, int n_cut, int ntri)
{
    const long nclen = 2L * nc10 + 1, M = nc10 + 1 - n_cut, N = nclen - 2L * n_cut;
    if (M < 2 || N < 3) return 0;
    const size_t per_tri = sizeof(double) * ((size_t)M * N * 3 + (size_t)N * N);
    const size_t batch = std::max<size_t>(1, std::min<size_t>({(size_t)std::max(ntri, 1), ((size_t)256 << 20) / per_tri,
                                                               (size_t)65535}));
    return sizeof(double) * ((size_t)nclen * nclen + N + ntri + 16) + batch * per_tri + 16 * (size_t)N;
}

// Why the parameters cannot run on a lag width nc10 (nullptr: they can).
const char *cyl_bs_invalid(const amber_cuda_cylbs_params *p, int nc10, int have_mask_sums)
{
    const int nclen = 2 * nc10 + 1, M = nc10 + 1 - p->n_cut, N = nclen - 2 * p->n_cut;
    if (p->n_cut < 0 || M < 2 || N < 3) return "n_cut leaves no data";
    if (N > 3072) return "N above 3072";
    if (!(p->mabs_norm != 0.0)) return "mabs_norm must be non-zero";
    if (p->denominator != 0 && p->denominator != 1) return "denominator must be 0 (counts) or 1 (mask sums)";
    if (p->denominator == 1 && !have_mask_sums) return "the mask-sum normaliser needs a v2 run";
    return nullptr;
}

}  // namespace amber

using namespace amber;

extern "C" int amber_cuda_cyl_bs(amber_cuda_ctx *c, const amber_cuda_cylbs_params *p, const double *tri_div,
                                 double *out)
{
    if (!c || !p || !out) return AMBER_ERR_ARG;
    if (c->last_ntri <= 0 || c->nc10 < 0) return fail(c, AMBER_ERR_STATE, "cyl_bs: no triangles run yet");
    if (p->denominator == 1 && !c->last_v2)
        return fail(c, AMBER_ERR_STATE, "cyl_bs: the mask-sum normaliser needs a v2 run");
    const int nc10 = c->nc10, nclen = 2 * nc10 + 1;
    const int ncut = p->n_cut;
    const int M = nc10 + 1 - ncut, N = nclen - 2 * ncut;
    // N ≤ 3072: the twiddle table of the transforms sits in shared memory (16·N bytes of the 48 KB default)
    if (const char *why = cyl_bs_invalid(p, nc10, c->last_v2))
        return fail(c, AMBER_ERR_ARG, "cyl_bs: %s (n_cut %d, nc10 %d)", why, ncut, nc10);
    cudaSetDevice(c->device);
    const long ncsize = (long)nclen * nclen;
    const int ntri = c->last_ntri;
    int rc;
    const double2 *tw;
    if ((rc = twiddle_table(c, N, &tw))) return rc;
    // normalisers: the closed-form counts (one array for every triangle) or each triangle's mask sums
    std::vector<double> host_aux;
    host_aux.reserve((size_t)ncsize + N + ntri);
    if (p->denominator == 0)
        for (long i = 0; i < ncsize; ++i) host_aux.push_back((double)c->counts[i]);
    const size_t inv_off = host_aux.size();
    if (tri_div)
        for (int t = 0; t < ntri; ++t) {
            if (!(tri_div[t] != 0.0)) return fail(c, AMBER_ERR_ARG, "cyl_bs: triangle %d divisor is zero", t);
            host_aux.push_back(1.0 / tri_div[t]);
        }
    std::vector<double> win;
    if (p->window) {
        // Blackman–Nuttall, mfunc_winds.py:17-31
        const double a0 = 0.3635819, a1 = 0.4891775, a2 = 0.1365995, a3 = 0.0106411;
        for (int i = 0; i < N; ++i) {
            const double ph = 2.0 * M_PI * i / (N - 1);
            win.push_back(a0 - a1 * cos(ph) + a2 * cos(2.0 * ph) - a3 * cos(3.0 * ph));
        }
    }
    // per batch of triangles: d [b][M][N] + X [b][M][N] complex + out [b][N][N]
    const size_t per_tri = sizeof(double) * ((size_t)M * N * 3 + (size_t)N * N);
    const int batch = (int)std::max<size_t>(1, std::min<size_t>({(size_t)ntri, ((size_t)256 << 20) / per_tri,
                                                                  (size_t)65535}));  // grid y / z limit
    // regions in doubles, each rounded up to 4 (32 bytes) so the double2 array stays aligned
    auto up4 = [](size_t n) { return (n + 3) / 4 * 4; };
    const size_t off_d = up4(host_aux.size() + win.size());
    const size_t off_x = off_d + up4((size_t)M * N * batch);
    const size_t off_o = off_x + 2 * (size_t)M * N * batch;
    const size_t total = off_o + (size_t)N * N * batch;
    if ((rc = ensure(c, c->mixed_scratch, sizeof(double) * total, "cylindrical bispectrum scratch"))) return rc;
    double *aux = (double *)c->mixed_scratch.p;
    double *d_win = win.empty() ? nullptr : aux + host_aux.size();
    double *d = aux + off_d;
    double2 *X = (double2 *)(aux + off_x);
    double *o = aux + off_o;
    if (!host_aux.empty() || !win.empty()) {
        std::vector<double> h(host_aux);
        h.insert(h.end(), win.begin(), win.end());
        if ((rc = cuda_check(c, cudaMemcpyAsync(aux, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice,
                                                c->stream), "cyl_bs upload")))
            return rc;
    }
    const double *res = (const double *)c->results.p;  // [ntri][2][ncsize]
    const double L = (double)N * p->dnu_mhz * p->rc_prime;
    const double scale = pow(p->rc, 4.0) * L * L;
    for (int t0 = 0; t0 < ntri; t0 += batch) {
        const int nb = std::min(batch, ntri - t0);
        const double *num = res + (size_t)t0 * 2 * ncsize;
        const double *den = p->denominator == 0 ? aux : num + ncsize;
        const long den_stride = p->denominator == 0 ? 0 : 2 * ncsize;
        const double *inv = tri_div ? aux + inv_off + t0 : nullptr;
        cylbs_fold<<<dim3((unsigned)(((long)M * N + kT - 1) / kT), nb), kT, 0, c->stream>>>(
            num, 2 * ncsize, den, den_stride, inv, nc10, ncut, 1.0 / p->mabs_norm, d_win, d);
        cylbs_rows<<<dim3((unsigned)((N + kT - 1) / kT), M, nb), kT, sizeof(double2) * N, c->stream>>>(d, M, N, tw, X);
        cylbs_cols<<<dim3((unsigned)((N + kT - 1) / kT), N, nb), kT, sizeof(double2) * N, c->stream>>>(X, M, N, tw,
                                                                                                      scale, o);
        c->launches += 3;
        if ((rc = cuda_check(c, cudaGetLastError(), "cyl_bs launch"))) return rc;
        if ((rc = cuda_check(c, cudaMemcpyAsync(out + (size_t)t0 * N * N, o, sizeof(double) * (size_t)nb * N * N,
                                                cudaMemcpyDeviceToHost, c->stream), "cyl_bs download")))
            return rc;
        if ((rc = cuda_check(c, cudaStreamSynchronize(c->stream), "cyl_bs"))) return rc;
    }
    return AMBER_OK;
}
