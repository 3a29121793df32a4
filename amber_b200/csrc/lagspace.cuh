// Lag-space contraction plan, shared by the plain FP64 and the int8 tensor-core
// contractions (replaces the loop of 4_fbe/amber.c:234-283 / amber_v2.c:230-288).
//
// The reference adds, for every admissible channel triplet (p1, p2, p3), the
// pixel sum Σ_x D1[p1,x]·D2[p2,x]·D3[p3,x] into lag cell
// (Δ2, Δ3) = (p2 − p1 + nc10, p3 − p1 + nc10).  Written per anchor p1 that is
// T_p1 = (D1[p1] ∘ D3[window])ᵀ · D2[window]; indexed by lags instead of
// channels, the windows of all anchors line up, so the anchor sum becomes part
// of the contraction dimension:
//
//     L[Δ3, Δ2] = Σ_{p1, x} A_{p1}[Δ3, x] · B_{p1}[Δ2, x],
//     A_{p1}[Δ3, x] = w·D1[p1, x] · w·D3[p1 − nc10 + Δ3, x],
//     B_{p1}[Δ2, x] = w·D2[p1 − nc10 + Δ2, x],
//
// one GEMM with K = anchors × pixels whose accumulator is the lag array itself.
// Channel multiplicities w (0 for flagged channels, > 1 for channels listed
// more than once) weight the operands; rows outside [0, nc) are zero.
//
// Tiles.  Accumulator rows are Δ3 (128 per tile), columns Δ2 (N per tile).
// Small lag windows (nclen ≤ 64) put k = ⌊128/nclen⌋ consecutive anchors into
// one tile: row r = a·nclen + Δ3 holds anchor slot a, and B is the window of
// the first anchor widened to N = nclen + k − 1 rows, so slot a's lag is
// Δ2 = column − a.  Large windows (nclen > 128) use ⌈nclen/128⌉² tile pairs.
//
// Work units.  The pixels are cut into blocks of LS_BLOCK; a unit is a tile
// pair × an anchor block × a run of consecutive pixel blocks, run by one CTA,
// which leaves the unit's FP64 sums in a partial tile of its own
// [LS_ROWS][LS_ROWS].  ls_reduce then adds, per lag cell, the partial tiles of
// every unit (and slot) in a fixed order with a compensated accumulator.  The
// units of a job depend only on the job and the SM count, never on what else
// shares the launch, so every result is deterministic.
#pragma once

#include <vector>

#include "common.cuh"

namespace amber {

constexpr int LS_BLOCK = 256;  // pixels per block (the int8 path's exponent block)
constexpr int LS_ROWS = 128;   // accumulator rows and columns of one tile
constexpr int LS_SPAN = 256;   // most channel rows one unit stages (a TMA box height)

struct LsShape {
    int nc, nc10, nclen;
    int k;        // anchor slots per tile (1 unless nclen ≤ 64)
    int T;        // tiles per lag axis
    int AB, nab;  // anchor-block width in channels, number of anchor blocks
    long nblk;    // pixel blocks
    long bpu;     // pixel blocks per unit
    int V;        // units per (tile pair, anchor block)
    int rows(int t3) const;  // accumulator rows used by tile t3
    int cols(int t2) const;  // MMA width N of tile t2 (multiple of 16)
    int lag_cols(int t2) const;  // lag columns Δ2 of tile t2 (k > 1: nclen)
    int units() const { return T * T * nab * V; }
};

// min_bpu: fewest pixel blocks per unit (partial-tile traffic against work per unit);
// force_bpu > 0: exactly that many blocks per unit (the last unit of a job may hold fewer)
LsShape ls_shape(int nc, int nc10, long k_px, int sms, long min_bpu = 8, long force_bpu = 0);

// Blocks per unit that a chunk_px option asks for (0 = chosen by the planner)
inline long ls_force_bpu(int chunk_px) { return chunk_px > 0 ? (chunk_px + LS_BLOCK - 1) / LS_BLOCK : 0; }

// One unit as the kernels see it.
struct LsUnit {
    int job;
    short t3, t2;
    int ab;           // anchor block
    int b0, b1;       // pixel blocks [b0, b1)
    long tile;        // its partial tile in the launch's partial buffer
    double work;      // modelled cost (launch order: largest first)
};

// Host side of one job: shape, anchor groups of every anchor block (first channel of each
// group of k consecutive channels that holds at least one anchor), and its units.
struct LsJobPlan {
    LsShape s;
    std::vector<int> groups;      // concatenated over anchor blocks
    std::vector<int> group_off;   // nab + 1 offsets into groups
    long unit_base = 0;           // first partial tile of the job in its launch
};
void ls_plan_job(LsJobPlan &p, int nc, int nc10, long k_px, const std::vector<int> &weight, int sms,
                 long min_bpu = 8, long force_bpu = 0);
void ls_units(const LsJobPlan &p, int job, std::vector<LsUnit> &out);

// Device description of one job for ls_reduce.
struct LsReduceJob {
    const double *partial;  // the job's partial tiles [units][LS_ROWS][LS_ROWS]
    double *lag;            // FP64 lag array [nclen][nclen], row Δ2, column Δ3
    int nclen, k, T, nab, V;
};
// lag = Σ over units (and slots) of the partial tiles, compensated, fixed order; one launch for
// every job of a contraction launch.  The descriptors are copied into the context's job staging.
int ls_reduce(amber_cuda_ctx *c, const std::vector<LsReduceJob> &jobs);

}  // namespace amber
