// Internal declarations shared by the libamber_cuda translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <vector>

#include "../../include/amber_cuda.h"

namespace amber {

// A device allocation owned by the context; grows on demand, never shrinks
// until the context is destroyed.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

// One set of ring maps on a common Ng1 × Ng1 grid: maps[slot][ch][x], row
// stride kp elements (kp = Ng1² rounded up to 64).
struct MapSet {
    long ng = 0;
    long k = 0;
    long kp = 0;
    int nslots = 0;
    std::vector<int> ring_of_slot;
    int slot_of_ring[256];
};

struct Engine;  // request engine (engine.cu)

}  // namespace amber

struct amber_cuda_ctx {
    int device = 0;
    int precision = AMBER_PREC_FP64;
    size_t budget = 0;
    size_t held = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int chunk_px = 0;
    int tile_n = 0;                // mixed path: forced p3 tile width, 0 = autotuned
    std::map<int, int> tile_tuned; // autotuner: lag-window class (nclen rounded up to 8) → p3 tile width
    std::vector<std::pair<int, float>> tile_trials;  // autotuner trials run here: (class·100 + BN, ms)
    int num_sms = 148;
    std::string err;

    // grid (normalised on the device)
    long N1 = 0, nc = 0;
    double Du = 0;
    int flag_key = -1;
    amber::DevBuf grid;  // double2 [cell][nc]
    amber::DevBuf mask;  // double  [cell][nc] (0/1)

    // rings
    int Nr = 0;
    std::vector<double> ulow, uhigh, uavg;

    // channels
    int nc10 = -1;
    std::vector<int> uf;       // as given
    std::vector<int> weight;   // multiplicity per channel (length nc)
    std::vector<int> anchors;  // channels with weight > 0, ascending
    std::vector<int64_t> counts;  // closed-form numdnu, nclen²
    int64_t total_vcp = 0;
    amber::DevBuf d_weight, d_anchors;

    // twiddle tables e^{2πik/N}, per N
    std::map<long, amber::DevBuf> twiddles;

    // working buffers
    amber::DevBuf y;        // pass-1 intermediate
    amber::DevBuf maps_d;   // D maps (FP64 path: double; mixed path: split planes)
    amber::DevBuf maps_i;   // I maps (v2)
    amber::DevBuf partial;  // per-anchor/k-split partial lag tiles
    amber::DevBuf results;  // per-triangle FP64 lag arrays [ntri][2][nclen²]
    amber::DevBuf ring_lohi;
    amber::DevBuf misc;
    amber::DevBuf mixed_scratch;
    amber::DevBuf lagred;  // two-pass lag reduction: per-group sums and compensations
    amber::DevBuf jobdesc; // contraction job descriptors and work items
    amber::DevBuf lagtrial; // autotuner: lag array of a discarded trial run
    amber::DevBuf lsred;    // lag-space reduction: job descriptors
    void *stage = nullptr; // pinned host staging of the job descriptors
    size_t stage_bytes = 0;
    amber::Engine *engine = nullptr;  // batched requests, created on the first enqueue
    bool contracts_elsewhere = false; // an engine's child context: its jobs run in the owner's contraction

    // per-phase device timing of the last run (CUDA events on the launch stream)
    struct PhaseEv {
        int phase;  // 0 maps, 1 contraction kernel, 2 lag reduction
        cudaEvent_t a, b;
    };
    std::vector<PhaseEv> phase_ev;
    size_t phase_used = 0;
    double phase_ms[3] = {0, 0, 0};
    long launches = 0;     // our kernels launched during the last run
    long contractions = 0; // contraction-kernel launches during the last run
    bool fp64_abs = false; // FP64 path sums |products| (the error scale of the mixed path)

    // last run
    int last_ntri = 0;
    int last_v2 = 0;
    double last_products = 0;
    float last_ms = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t tev0 = nullptr, tev1 = nullptr;  // autotuner trials
};

namespace amber {

// Record a phase boundary on the context's stream (timing of the last run).
void phase_begin(amber_cuda_ctx *c, int phase);
void phase_end(amber_cuda_ctx *c);

int fail(amber_cuda_ctx *c, int code, const char *fmt, ...);
int cuda_check(amber_cuda_ctx *c, cudaError_t e, const char *what);
int ensure(amber_cuda_ctx *c, DevBuf &b, size_t bytes, const char *what);
int twiddle_table(amber_cuda_ctx *c, long n, const double2 **out);

// Map builder: ring-mask + unnormalised c2r of every channel of the given
// rings onto an ng × ng grid.  src_complex: double2 grid; else real mask.
// Writes FP64 maps (out_f64) or split-BF16 hi/lo planes (out_hi/out_lo)
// with row stride kp.  chan_base/nch select source channels.
struct MapJob {
    const void *src;
    bool src_complex;
    long n1, nc;         // source grid side and channel count
    long chan_base, nch; // source channel window
    long ng, kp;         // output side and row stride
    int nslots;
    const double *lohi;  // device: lo[s], hi[s] interleaved
    std::vector<double> lo, hi;  // host copies
    double *out_f64;
    uint16_t *out_hi, *out_lo;  // bf16 planes
    float *out_f32;               // mixed path: maps weighted by the channel multiplicities
    const int *weight;            // device multiplicities of the source channels (mixed path)
    int8_t *dig;                  // mixed path: digit planes [slot][3][kp/16][nch][16] (kp multiple of 256)
    int *bexp;                    // mixed path: exponent per (slot, 256-pixel block)
};
int build_maps(amber_cuda_ctx *c, const MapJob &job);

// FP64 contraction of one triangle into a lag array (device).
int contract_fp64(amber_cuda_ctx *c, const double *m1, const double *m2, const double *m3, long k, long kp,
                  double *lag_out);
// One FP64 contraction job (one triangle's D or mask pass on the context's channels).
struct F64Job {
    const double *m1, *m2, *m3;  // [nc][kp] maps of r1, r2, r3
    long k, kp;
    double *lag_out;             // device FP64 lag array [nclen²]
};
// All jobs in as few launches as the partial-tile memory allows, then one reduction per launch.
int contract_fp64_jobs(amber_cuda_ctx *c, const std::vector<F64Job> &jobs);
// Split-BF16×3 contraction (tcgen05, FP32 accumulation in TMEM).
int contract_bf16x3(amber_cuda_ctx *c, const uint16_t *h1, const uint16_t *l1, const uint16_t *h2,
                    const uint16_t *l2, const uint16_t *h3, const uint16_t *l3, long k, long kp, double *lag_out);
// Mixed-precision contraction: base-254 int8 digits on the tensor cores
// (tcgen05 kind::i8, exact int32 accumulation in TMEM).
struct DigitMaps {
    const float *f32;                 // [nc][kp], weighted by the channel multiplicities
    const int8_t *dig;                // [3][kp/16][nc][16] base-254 digits of f32
    const int *bexp;                  // [kp/256] block exponents
};
int contract_i8(amber_cuda_ctx *c, const DigitMaps &m1, const DigitMaps &m2, const DigitMaps &m3, long k, long kp,
                double *lag_out);
// One mixed-precision contraction job: one triangle's D or mask pass of one realisation.
struct I8Job {
    DigitMaps m1, m2, m3;   // ring maps of r1, r2, r3 on the job's Ng1 grid
    long k, kp;             // pixels, row stride (a multiple of 256)
    int nc, nc10;           // the realisation's channel count and lag half-width
    const std::vector<int> *weight;  // host: channel multiplicities (the planner's anchor groups)
    int nanchors;
    bool mask_pass;         // sampling-mask maps: four product digits (a second sweep for class 3)
    double *lag_out;        // device: FP64 lag array [nclen²]
};
// All jobs in as few persistent launches as the partial-tile memory allows (jobs of
// different realisations may share a launch); each job's result depends on the job only.
int contract_i8_jobs(amber_cuda_ctx *c, const std::vector<I8Job> &jobs);

// One realisation's list of triangles, run in map-set batches: the triangles are grouped
// by r1 (one Ng1 grid per group) and each group is cut into batches whose ring maps fit
// the context's budget.
struct RunState {
    struct Group {
        int r1;
        long ng;
        std::vector<int> tris;  // indices into tri
    };
    std::vector<int> tri;  // 3 rings per triangle
    int want_v2 = 0;
    std::vector<Group> groups;
    size_t gi = 0, ti = 0;  // next group, next triangle in it
};
int run_begin(amber_cuda_ctx *c, RunState &st, int ntri, const int *tri, int want_v2);
// Builds the ring maps of the next batch.  Mixed precision: appends the batch's jobs to
// *jobs for the caller to contract (or contracts them at once when jobs is null); other
// precisions contract here.  Returns 1 after a batch, 0 when the run is complete, <0 on error.
int run_next_batch(amber_cuda_ctx *c, RunState &st, std::vector<I8Job> *jobs);
// Device bytes of one ring slot of a map batch on an ng grid (D and, for v2, mask maps,
// plus the map builder's intermediate).
size_t map_slot_bytes(int precision, long ng, long nc, int want_v2);
// Ng1 of a ring (amber.c:193-197) and calCR's closed triangles (r1 ≥ r2 ≥ r3, in its order).
long ring_ng1(double uhigh, double du);
std::vector<int> closed_triangles(const std::vector<double> &ulow, const std::vector<double> &uhigh);
// Stops the context's request engine (pending requests finish, queued ones are dropped).
void engine_shutdown(amber_cuda_ctx *c);
// lag[d] = Σ_u partial[u][d] (compensated, fixed order); accumulate adds to lag[d].
int lag_reduce(amber_cuda_ctx *c, const double *partial, long nunits, long ncsize, double *lag,
               bool accumulate = false);
// Device bytes the mixed-precision contraction keeps for the partial tiles of one launch.
size_t contract_partial_cap(const amber_cuda_ctx *c);

// amber_cuda_cyl_bs: device bytes it may add to a context, and why parameters cannot
// run on a lag width (nullptr: they can).
size_t cyl_bs_bytes(int nc10, int n_cut, int ntri);
const char *cyl_bs_invalid(const amber_cuda_cylbs_params *p, int nc10, int have_mask_sums);
// Σ_x a·b·c over n points (FP64, deterministic) into out[0].
// calCR: Num of every triangle (r1, r2, r3 in tri) from the N1² mask maps [ring][n], into device out[t].
int triple_sums(amber_cuda_ctx *c, const double *maps, long n, const std::vector<int> &tri, double *out);

}  // namespace amber
