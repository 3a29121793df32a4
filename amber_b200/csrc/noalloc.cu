// Allocation-free FP64 lag contraction of one triangle.
//
// Some callers own every byte of device memory themselves: a host process
// that reserves its whole HBM budget at start-up and hands slices of it out,
// or an application whose own caching allocator must stay the only thing
// that allocates on the device.  Such callers cannot let a library call
// cudaMalloc, which the context-based entry points do for their maps and
// partial tiles.  This entry point takes the three ring-map sets and the
// output lag array as device pointers the caller already owns, and keeps its
// only scratch — the FP64 partial lag tiles and the channel tables — in one
// file-scope __device__ array of fixed size (every GPU that loads the library
// holds it until the process exits).  It calls no cudaMalloc, cudaFree or
// allocating library routine.
//
// The arithmetic is the plain FP64 path's (the reference loop of
// 4_fbe/amber.c:247-279 restated in FP64): 64 × 64 tiles of one anchor's lag
// window over a pixel range, weighted by the channel multiplicities, then a
// compensated fixed-order sum per lag cell.  Anchors are processed in batches
// whose partial tiles fit the scratch; each batch's compensated sum is added
// to the output in batch order, so results are deterministic.
#include <stdio.h>

#include <algorithm>
#include <mutex>

#include <cuda.h>

#include "common.cuh"

namespace {

constexpr long kScratchDoubles = 1L << 20;  // 8 MiB in total
constexpr int kMaxChannels = 4096;           // channel tables: weights + anchors, at the tail
constexpr long kTableDoubles = (2L * kMaxChannels * sizeof(int) + sizeof(double) - 1) / sizeof(double);
constexpr long kPartialDoubles = kScratchDoubles - kTableDoubles;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int TT = 64;
constexpr int KB = 16;

__global__ void __launch_bounds__(256) noalloc_tile_kernel(const double *__restrict__ m1,
                                                            const double *__restrict__ m2,
                                                            const double *__restrict__ m3, long k, long kp,
                                                            const int *__restrict__ anchors, int a_first,
                                                            const int *__restrict__ weight, int nc, int nc10,
                                                            int tiles, long kchunk, double *__restrict__ partial)
{
    __shared__ __align__(16) double As[KB][TT + 2];
    __shared__ __align__(16) double Bs[KB][TT + 2];
    __shared__ int prow[TT], pcol[TT];
    const int tid = threadIdx.x;
    const int a = blockIdx.y, ks = blockIdx.z, KS = gridDim.z;
    const int t2 = blockIdx.x / tiles, t3 = blockIdx.x % tiles;
    const int p1 = anchors[a_first + a];
    const int nclen = 2 * nc10 + 1;
    const int d2b = TT * t2, d3b = TT * t3;
    const int tx = tid & 15, ty = tid >> 4;
    double *out = partial + ((size_t)a * KS + ks) * nclen * nclen;
    if (tid < TT) {
        const int d = d2b + tid, p = p1 - nc10 + d;
        prow[tid] = (d < nclen && p >= 0 && p < nc && weight[p] > 0) ? p : -1;
    } else if (tid < 2 * TT) {
        const int d = d3b + tid - TT, p = p1 - nc10 + d;
        pcol[tid - TT] = (d < nclen && p >= 0 && p < nc && weight[p] > 0) ? p : -1;
    }
    __syncthreads();
    double acc[4][4] = {};
    const long x0 = (long)ks * kchunk, x1 = min(k, x0 + kchunk);
    const double *c1 = m1 + (long)p1 * kp;
    for (long xs = x0; xs < x1; xs += KB) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int e = tid + i * 256, r = e / KB, xx = e % KB;
            const long x = xs + xx;
            double va = 0.0, vb = 0.0;
            if (x < x1) {
                if (prow[r] >= 0) va = c1[x] * m2[(long)prow[r] * kp + x];
                if (pcol[r] >= 0) vb = m3[(long)pcol[r] * kp + x];
            }
            As[xx][r] = va;
            Bs[xx][r] = vb;
        }
        __syncthreads();
#pragma unroll
        for (int xx = 0; xx < KB; ++xx) {
            double av[4], bv[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                av[i] = As[xx][ty * 4 + i];
                bv[i] = Bs[xx][tx * 4 + i];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }
    const double w1 = (double)weight[p1];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = ty * 4 + i, d2 = d2b + r;
        if (d2 >= nclen) continue;
        const double wr = prow[r] >= 0 ? w1 * (double)weight[prow[r]] : 0.0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int cc = tx * 4 + j, d3 = d3b + cc;
            if (d3 >= nclen) continue;
            const double wc = pcol[cc] >= 0 ? (double)weight[pcol[cc]] : 0.0;
            out[(long)d2 * nclen + d3] = acc[i][j] * wr * wc;
        }
    }
}

// lag[d] (+)= Σ_{u < nunits} partial[u][d], TwoSum-compensated, fixed order.
__global__ void noalloc_batch_sum(const double *__restrict__ partial, long nunits, long ncsize, int accumulate,
                                  double *__restrict__ lag)
{
    const long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= ncsize) return;
    double s = 0.0, comp = 0.0;
    for (long u = 0; u < nunits; ++u) {
        const double v = partial[u * ncsize + d];
        const double t = s + v, bp = t - s;
        comp += (s - (t - bp)) + (v - bp);
        s = t;
    }
    s += comp;
    lag[d] = accumulate ? lag[d] + s : s;
}

// Device address of the scratch array, looked up once per device and context: a context
// destroyed and recreated (cudaDeviceReset) maps the array anew, so the cached address is
// kept together with the context it belongs to and looked up again when that changes.
std::mutex g_mutex;
double *g_scratch_ptr[64] = {};
CUcontext g_scratch_ctx[64] = {};

}  // namespace

extern "C" int amber_cuda_contract_fp64_noalloc(const double *d_m1, const double *d_m2, const double *d_m3, long nc,
                                                long k, long kp, int nc10, const int *weight, double *d_lag,
                                                void *stream, char *err_msg, size_t err_len)
{
    auto reject = [&](int code, const char *msg) {
        if (err_msg && err_len) snprintf(err_msg, err_len, "%s", msg);
        return code;
    };
    if (!d_m1 || !d_m2 || !d_m3 || !d_lag || !weight) return reject(AMBER_ERR_ARG, "NULL pointer argument");
    if (nc <= 0 || nc > kMaxChannels) return reject(AMBER_ERR_ARG, "nc outside [1, 4096]");
    if (k <= 0 || kp < k) return reject(AMBER_ERR_ARG, "need 0 < k <= kp");
    if (nc10 < 0 || nc10 >= nc) return reject(AMBER_ERR_ARG, "nc10 outside [0, nc)");
    const int nclen = 2 * nc10 + 1;
    const long ncsize = (long)nclen * nclen;
    if (ncsize > kPartialDoubles)
        return reject(AMBER_ERR_ARG, "lag window too large for the 8 MiB scratch (nclen^2 must be <= 1044480, nc10 <= 510)");

    cudaStream_t s = (cudaStream_t)stream;
    // The channel tables below are copied from a host buffer that lives only for this call.
    // A stream under capture would record that copy for later replays instead of making it
    // now, so a capturing stream is refused.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
        cudaGetLastError();
        return reject(AMBER_ERR_ARG, "invalid stream");
    }
    if (cap != cudaStreamCaptureStatusNone)
        return reject(AMBER_ERR_ARG, "stream is being captured: this call uploads host channel tables when it is made");

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return reject(AMBER_ERR_NODEV, "no device");
    double *scratch;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        // cudaGetDevice does not initialise the device's primary context; cudaSetDevice does
        // and makes it current, so that the context handle below exists
        if (cudaSetDevice(dev) != cudaSuccess) {
            cudaGetLastError();
            return reject(AMBER_ERR_NODEV, "cannot make the device current");
        }
        // the driver call is resolved through the runtime, so the library needs no link-time libcuda
        static CUresult (*ctx_current)(CUcontext *) = nullptr;
        if (!ctx_current) {
            void *fn = nullptr;
            cudaDriverEntryPointQueryResult q;
            if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn)
                return reject(AMBER_ERR_CUDA, "cuCtxGetCurrent unavailable");
            ctx_current = (CUresult(*)(CUcontext *))fn;
        }
        CUcontext ctx = nullptr;
        if (ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return reject(AMBER_ERR_CUDA, "no current context");
        if (!g_scratch_ptr[dev] || g_scratch_ctx[dev] != ctx) {
            void *p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                cudaGetLastError();
                return reject(AMBER_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
            }
            g_scratch_ptr[dev] = (double *)p;
            g_scratch_ctx[dev] = ctx;
        }
        scratch = g_scratch_ptr[dev];
    }

    // channel tables (host → the scratch's tail): multiplicities and the anchors (channels with weight > 0)
    int table[2 * kMaxChannels];
    int na = 0;
    for (long p = 0; p < nc; ++p) {
        if (weight[p] < 0) return reject(AMBER_ERR_ARG, "negative channel multiplicity");
        table[p] = weight[p];
        if (weight[p] > 0) table[nc + na++] = (int)p;
    }
    int *d_table = reinterpret_cast<int *>(scratch + kPartialDoubles);
    if (cudaMemcpyAsync(d_table, table, sizeof(int) * (nc + (na > 0 ? na : 1)), cudaMemcpyHostToDevice, s) !=
        cudaSuccess) {
        cudaGetLastError();
        return reject(AMBER_ERR_CUDA, "channel table upload failed");
    }
    if (na == 0) {
        if (cudaMemsetAsync(d_lag, 0, sizeof(double) * ncsize, s) != cudaSuccess) {
            cudaGetLastError();
            return reject(AMBER_ERR_CUDA, "clearing the lag array failed");
        }
        return AMBER_OK;
    }
    const int tiles = (nclen + TT - 1) / TT;
    // units per batch that fit the partial area; k-split to fill the GPU when anchors are few
    const long cap_units = kPartialDoubles / ncsize;
    int KS = (int)std::max<long>(1, std::min<long>(cap_units / std::max(1, na), (k + 1023) / 1024));
    KS = std::min(KS, 8);
    const long kchunk = ((k + KS - 1) / KS + KB - 1) / KB * KB;
    KS = (int)((k + kchunk - 1) / kchunk);
    const int batch = (int)std::max<long>(1, cap_units / KS);
    for (int a0 = 0; a0 < na; a0 += batch) {
        const int nb = std::min(batch, na - a0);
        dim3 grid((unsigned)(tiles * tiles), (unsigned)nb, (unsigned)KS);
        noalloc_tile_kernel<<<grid, 256, 0, s>>>(d_m1, d_m2, d_m3, k, kp, d_table + nc, a0, d_table, (int)nc, nc10,
                                                 tiles, kchunk, scratch);
        noalloc_batch_sum<<<(unsigned)((ncsize + 255) / 256), 256, 0, s>>>(scratch, (long)nb * KS, ncsize, a0 > 0,
                                                                          d_lag);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return reject(AMBER_ERR_CUDA, cudaGetErrorString(e));
    return AMBER_OK;
}
