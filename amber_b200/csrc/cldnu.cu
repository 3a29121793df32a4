// MAPS two-point function on the device: the multi-frequency angular power
// spectrum C_ℓ(Δν) of the normalised grid, as 4_fbe/maps.c:179-210 computes it
// by calling cl_dnu (4_fbe/amber_funcs.c:1418-1488) for every channel pair
// nn1 <= nn2.  Per log bin b of U = |(ia, j)|·Du in [umin, umax) and pair (p, q):
//   no_b[p]     = Σ_{cells in b} NTiG[p]
//   S_b[p][q]   = Σ_{cells in b} (Re_p·Re_q + Im_p·Im_q)·NTiG[p]
//   binps       = S_b[p][q] / no_b[p]                  (where no_b[p] != 0)
//   cldnu[b][Δ] = Σ_{p = 0 .. nc−1−Δ} binps(p, p + Δ)  (p ascending)
// and the printed binu / num are usum / no and no of the last pair (p = nc−1).
//
// Every sum runs in the reference's order with the reference's roundings
// (cells in index order, separate multiplies and adds — the reference build has
// no FMA contraction — then the division, then the Δ sums over p ascending), so
// the results are bit-identical to the reference's loops.  The bin of each cell
// (sqrt, log10, floor of the reference's expressions) is computed on the host
// with the C library, so no device-vs-host libm difference can move a cell.
//
// Kernels:
//   cldnu_norm   one thread per (bin, channel): no_b[p], usum_b[p];
//   cldnu_pairs  one CTA per (bin, 32×32 tile of (p, q) with q-tile >= p-tile):
//                the bin's cells in chunks of 16 staged through shared memory,
//                4×4 (p, q) per thread, FP64; writes binps to P[b][p][q − p];
//   cldnu_reduce one thread per (bin, Δ): Σ_p P[b][p][Δ].
// Work: 5 FP64 operations per (cell, pair); the bin's grid rows are read once
// per tile pair.  FP64-pipe bound; tiny next to the bispectrum.
#include <math.h>

#include <algorithm>
#include <vector>

#include "common.cuh"

namespace amber {

namespace {

constexpr int kTile = 32;   // (p, q) tile
constexpr int kChunk = 16;  // cells per shared-memory stage

__global__ void cldnu_norm(const double *__restrict__ mask, const int *__restrict__ cells,
                           const double *__restrict__ uu, const int *__restrict__ bin_off, long nc,
                           int *__restrict__ no, double *__restrict__ usum)
{
    const int b = blockIdx.y;
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nc) return;
    int n = 0;
    double u = 0.0;
    for (int k = bin_off[b]; k < bin_off[b + 1]; ++k) {
        const double w = mask[(long)cells[k] * nc + p];
        n = (int)((double)n + w);  // no[tmp] += NTiG (int += double)
        u = __dadd_rn(u, __dmul_rn(uu[k], w));
    }
    no[(long)b * nc + p] = n;
    usum[(long)b * nc + p] = u;
}

__global__ void __launch_bounds__(64) cldnu_pairs(const double2 *__restrict__ grid, const double *__restrict__ mask,
                                                  const int *__restrict__ cells, const int *__restrict__ bin_off,
                                                  const int *__restrict__ no, long nc, int ntile,
                                                  double *__restrict__ P)
{
    __shared__ double sre1[kChunk][kTile], sim1[kChunk][kTile], sw1[kChunk][kTile];
    __shared__ double sre2[kChunk][kTile], sim2[kChunk][kTile];
    const int b = blockIdx.y;
    // blockIdx.x → (tp, tq), tq >= tp
    int t = blockIdx.x, tp = 0;
    while (t >= ntile - tp) {
        t -= ntile - tp;
        ++tp;
    }
    const int tq = tp + t;
    const long p0 = (long)tp * kTile, q0 = (long)tq * kTile;
    const int tx = threadIdx.x & 7, ty = threadIdx.x >> 3;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
    const int k0 = bin_off[b], k1 = bin_off[b + 1];
    for (int kc = k0; kc < k1; kc += kChunk) {
        const int nk = min(kChunk, k1 - kc);
        __syncthreads();
        for (int e = threadIdx.x; e < kChunk * kTile; e += blockDim.x) {
            const int k = e / kTile, ch = e % kTile;
            double r1 = 0, i1 = 0, w1 = 0, r2 = 0, i2 = 0;
            if (k < nk) {
                const long cell = cells[kc + k];
                if (p0 + ch < nc) {
                    const double2 g = grid[cell * nc + p0 + ch];
                    r1 = g.x;
                    i1 = g.y;
                    w1 = mask[cell * nc + p0 + ch];
                }
                if (q0 + ch < nc) {
                    const double2 g = grid[cell * nc + q0 + ch];
                    r2 = g.x;
                    i2 = g.y;
                }
            }
            sre1[k][ch] = r1;
            sim1[k][ch] = i1;
            sw1[k][ch] = w1;
            sre2[k][ch] = r2;
            sim2[k][ch] = i2;
        }
        __syncthreads();
        for (int k = 0; k < nk; ++k) {
            double r1[4], i1[4], w1[4], r2[4], i2[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                r1[i] = sre1[k][ty + 8 * i];
                i1[i] = sim1[k][ty + 8 * i];
                w1[i] = sw1[k][ty + 8 * i];
                r2[i] = sre2[k][tx + 8 * i];
                i2[i] = sim2[k][tx + 8 * i];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    // numer = Re1·Re2 + Im1·Im2; numer *= NTiG; pksum += numer
                    const double numer = __dmul_rn(__dadd_rn(__dmul_rn(r1[i], r2[j]), __dmul_rn(i1[i], i2[j])), w1[i]);
                    acc[i][j] = __dadd_rn(acc[i][j], numer);
                }
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const long p = p0 + ty + 8 * i;
        if (p >= nc) continue;
        const int n = no[(long)b * nc + p];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const long q = q0 + tx + 8 * j;
            if (q < p || q >= nc) continue;
            P[((long)b * nc + p) * nc + (q - p)] = n != 0 ? __ddiv_rn(acc[i][j], (double)n) : acc[i][j];
        }
    }
}

__global__ void cldnu_reduce(const double *__restrict__ P, long nc, double *__restrict__ cldnu)
{
    const int b = blockIdx.y;
    const long d = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= nc) return;
    double s = 0.0;
    for (long p = 0; p + d < nc; ++p) s = __dadd_rn(s, P[((long)b * nc + p) * nc + d]);
    cldnu[(long)b * nc + d] = s;
}

}  // namespace

}  // namespace amber

using namespace amber;

extern "C" int amber_cuda_cl_dnu(amber_cuda_ctx *c, int NB, double umin, double umax, double *cldnu, double *numdnu,
                                 double *binu, int *num)
{
    if (!c || !cldnu) return AMBER_ERR_ARG;
    if (!c->grid.p || c->N1 <= 0 || c->nc <= 0) return fail(c, AMBER_ERR_STATE, "cl_dnu: no grid loaded");
    if (NB <= 0 || NB > 4096 || !(umin > 0) || !(umax > umin))
        return fail(c, AMBER_ERR_ARG, "cl_dnu: need 0 < NB <= 4096 and 0 < umin < umax");
    const long N1 = c->N1, H = N1 / 2 + 1, nc = c->nc;
    // bins of the cells, the reference's expressions (amber_funcs.c:1448-1462) on the host
    const double binsiz = log10(umax / umin) / (1. * NB);
    std::vector<std::vector<int>> by_bin(NB);
    std::vector<std::vector<double>> uu_bin(NB);
    for (long i = 0; i < N1; ++i)
        for (long j = 0; j < H; ++j) {
            const long ia = (i > N1 / 2) ? (N1 - i) : i;
            const double uu = sqrt(1. * (ia * ia + j * j)) * c->Du;
            if (!(uu >= umin && uu < umax)) continue;
            const int tmp = (int)floor(log10(uu / umin) / binsiz);
            if (tmp < 0 || tmp >= NB) continue;  // U rounding onto umax: the reference writes past its arrays
            by_bin[tmp].push_back((int)(i * H + j));
            uu_bin[tmp].push_back(uu);
        }
    std::vector<int> cells, off(NB + 1, 0);
    std::vector<double> uus;
    for (int b = 0; b < NB; ++b) {
        cells.insert(cells.end(), by_bin[b].begin(), by_bin[b].end());
        uus.insert(uus.end(), uu_bin[b].begin(), uu_bin[b].end());
        off[b + 1] = (int)cells.size();
    }
    const long ncell = std::max<long>(1, (long)cells.size());
    const int ntile = (int)((nc + kTile - 1) / kTile);
    // scratch: P [NB][nc][nc] + usum [NB][nc] + uu [cells] (doubles), then no [NB][nc] + cells + off (ints)
    auto up4 = [](size_t n) { return (n + 3) / 4 * 4; };
    const size_t nP = (size_t)NB * nc * nc, nU = (size_t)NB * nc;
    const size_t o_usum = up4(nP), o_uu = o_usum + up4(nU), o_int = o_uu + up4(ncell);
    const size_t n_int = (size_t)NB * nc + ncell + NB + 1;
    const size_t bytes = sizeof(double) * o_int + sizeof(int) * n_int;
    int rc;
    if ((rc = ensure(c, c->mixed_scratch, bytes, "cl_dnu scratch"))) return rc;
    cudaSetDevice(c->device);
    double *P = (double *)c->mixed_scratch.p;
    double *usum = P + o_usum, *d_uu = P + o_uu;
    int *no = (int *)(P + o_int), *d_cells = no + (size_t)NB * nc, *d_off = d_cells + ncell;
    cudaStream_t s = c->stream;
    if (!cells.empty()) {
        if ((rc = cuda_check(c, cudaMemcpyAsync(d_cells, cells.data(), sizeof(int) * cells.size(),
                                                cudaMemcpyHostToDevice, s), "cl_dnu cells")))
            return rc;
        if ((rc = cuda_check(c, cudaMemcpyAsync(d_uu, uus.data(), sizeof(double) * uus.size(), cudaMemcpyHostToDevice,
                                                s), "cl_dnu U")))
            return rc;
    }
    if ((rc = cuda_check(c, cudaMemcpyAsync(d_off, off.data(), sizeof(int) * (NB + 1), cudaMemcpyHostToDevice, s),
                         "cl_dnu bins")))
        return rc;
    const double2 *grid = (const double2 *)c->grid.p;
    const double *mask = (const double *)c->mask.p;
    cldnu_norm<<<dim3((unsigned)((nc + 127) / 128), NB), 128, 0, s>>>(mask, d_cells, d_uu, d_off, nc, no, usum);
    cldnu_pairs<<<dim3((unsigned)(ntile * (ntile + 1) / 2), NB), 64, 0, s>>>(grid, mask, d_cells, d_off, no, nc,
                                                                             ntile, P);
    // no / usum come back first; the Δ sums then reuse the usum slot (same stream, in order)
    std::vector<int> h_no((size_t)NB * nc);
    std::vector<double> h_usum((size_t)NB * nc);
    if ((rc = cuda_check(c, cudaGetLastError(), "cl_dnu launch"))) return rc;
    if ((rc = cuda_check(c, cudaMemcpyAsync(h_no.data(), no, sizeof(int) * h_no.size(), cudaMemcpyDeviceToHost, s),
                         "cl_dnu counts")))
        return rc;
    if ((rc = cuda_check(c, cudaMemcpyAsync(h_usum.data(), usum, sizeof(double) * h_usum.size(), cudaMemcpyDeviceToHost,
                                            s), "cl_dnu U sums")))
        return rc;
    cldnu_reduce<<<dim3((unsigned)((nc + 127) / 128), NB), 128, 0, s>>>(P, nc, usum);
    c->launches += 3;
    if ((rc = cuda_check(c, cudaGetLastError(), "cl_dnu launch"))) return rc;
    if ((rc = cuda_check(c, cudaMemcpyAsync(cldnu, usum, sizeof(double) * nU, cudaMemcpyDeviceToHost, s),
                         "cl_dnu download")))
        return rc;
    if ((rc = cuda_check(c, cudaStreamSynchronize(s), "cl_dnu"))) return rc;
    // maps.c:187 (numdnu[nn2−nn1] += 1 per pair) and the last pair's binu / num (maps.c:197-205)
    if (numdnu)
        for (long d = 0; d < nc; ++d) {
            double v = 0.;
            for (long p = 0; p + d < nc; ++p) v += 1.;
            numdnu[d] = v;
        }
    for (int b = 0; b < NB; ++b) {
        const int n = h_no[(size_t)b * nc + nc - 1];
        const double u = h_usum[(size_t)b * nc + nc - 1];
        if (binu) binu[b] = n != 0 ? u / (1. * n) : u;
        if (num) num[b] = n;
    }
    return AMBER_OK;
}
