/*
 * libamber_cuda — B200 (sm_100a) implementation of the AMBER estimator hot
 * path behind a plain C ABI: no CUDA or torch types in any signature, host
 * pointers and sizes only.  A C driver (amber_gpu) links it as a drop-in for
 * the per-triangle loop of 4_fbe/amber.c and 4_fbe/amber_v2.c, and the
 * Python package loads it with ctypes.
 *
 * Ownership: the context owns every device allocation; host buffers always
 * belong to the caller.  One context per host thread; calls on one context
 * are not re-entrant.  Every call returns AMBER_OK (0) or a negative status
 * and never exits the process; amber_cuda_last_error() explains the last
 * failure.  All calls are synchronous from the caller's point of view.
 */
#ifndef AMBER_CUDA_H
#define AMBER_CUDA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define AMBER_API __attribute__((visibility("default")))
#else
#define AMBER_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define AMBER_OK 0
#define AMBER_ERR_ARG (-1)      /* bad argument (size, range, NULL) */
#define AMBER_ERR_OOM (-2)      /* device allocation failed or over the HBM budget */
#define AMBER_ERR_CUDA (-3)     /* CUDA runtime or kernel launch error */
#define AMBER_ERR_TIMEOUT (-4)  /* a bounded device-side wait gave up */
#define AMBER_ERR_OVERFLOW (-5) /* a count does not fit the output type (v1 numdnu is int32) */
#define AMBER_ERR_STATE (-6)    /* call order: grid / rings / channels not set yet */
#define AMBER_ERR_NODEV (-7)    /* no usable sm_100 device: the library has no CPU fallback */

/* ---- precision of the triple-product contraction ---- */
#define AMBER_PREC_FP64 0   /* plain FP64 restatement of the reference loop (CUDA cores) */
#define AMBER_PREC_MIXED 1  /* int8 tensor cores: base-254 fixed-point digits, exact int32 accumulation in TMEM,
                               FP64 recombination and compensated lag reduction (≤1e-6 of Σ|products|) */
#define AMBER_PREC_BF16X3 2 /* split-BF16×3 on the tensor cores with FP32 accumulation in TMEM; kept for
                               comparison: it misses 1e-6 on coherent v2 sampling-mask sums */
#define AMBER_PREC_FP64_ABS 3 /* the FP64 path summing |products|: the per-lag-cell scale against which
                                 the mixed path's error is measured (no reference counterpart) */

typedef struct amber_cuda_ctx amber_cuda_ctx;

typedef struct amber_cuda_opts {
    int device;            /* CUDA device ordinal */
    int precision;         /* AMBER_PREC_FP64 or AMBER_PREC_MIXED */
    size_t hbm_budget;     /* max device bytes the context may hold; 0 = 90 % of free memory */
    void *stream;          /* optional cudaStream_t to launch on (NULL = the context's own stream) */
    int chunk_px;          /* lag-space contraction (mixed and FP64): pixels per work unit, i.e. per partial
                              lag tile summed in FP64, rounded up to whole 256-pixel blocks; 0 = chosen by the
                              planner (about six units per SM).  It sets only the FP64 summation grouping. */
    int tile_n;            /* accepted for compatibility (0, 32, 64 or 128) and ignored: the lag-space
                              contraction has no tile width to choose */
} amber_cuda_opts;

AMBER_API void amber_cuda_default_opts(amber_cuda_opts *opts);
AMBER_API int amber_cuda_create(const amber_cuda_opts *opts, amber_cuda_ctx **out);
AMBER_API void amber_cuda_destroy(amber_cuda_ctx *ctx);
AMBER_API const char *amber_cuda_last_error(const amber_cuda_ctx *ctx);

/* ---- grid input: replaces initialize + ReadGVnAC_gridding + normalize_data
 * (4_fbe/amber_funcs.c:1720-1779, 1861-1941, 1946-1978).  The summed grid and
 * the sampling counts are uploaded and normalised on the device:
 * GV /= NTiG where NTiG > 0, then NTiG := 1 there.
 * Packed form: re_im[(cell·nc + ch)·2 + {0,1}], ntig[cell·nc + ch] with
 * cell = ii·(N1/2+1) + jj — exactly the order of the GV_data / sampling files.
 * Pointer-per-cell form: the reference's own double** arrays
 * (amber_funcs.c:1756-1769), GVre[cell][ch] etc. */
AMBER_API int amber_cuda_load_grid_packed(amber_cuda_ctx *ctx, long N1, long nc, double Du, int flag_key,
                                const double *re_im, const double *ntig);
AMBER_API int amber_cuda_load_grid(amber_cuda_ctx *ctx, long N1, long nc, double Du, int flag_key,
                         const double *const *GVre, const double *const *GVim, const double *const *NTiG);
/* The packed form with re_im and ntig already in device memory on the context's device (a cube
 * kept resident between estimates): normalised straight from there, nothing is copied in. */
AMBER_API int amber_cuda_load_grid_device(amber_cuda_ctx *ctx, long N1, long nc, double Du, int flag_key,
                                          const double *re_im, const double *ntig);

/* ---- ring edges: replaces annular_rings (amber_funcs.c:2022-2094).  Uavg is
 * computed as in amber_funcs.c:2065.  Rings must lie inside the grid
 * (UHigh ≤ N1/2), otherwise the reference would index outside it. */
AMBER_API int amber_cuda_set_rings(amber_cuda_ctx *ctx, int Nr, const double *ULow, const double *UHigh);
AMBER_API int amber_cuda_get_uavg(const amber_cuda_ctx *ctx, double *Uavg);

/* ---- channels: replaces get_uf_chans + precompute_unflg_vcp /
 * precompute_vcp_dnu (amber_funcs.c:2485-2508, 2207-2259, 2264-2310).
 * uf_nc == 0 means flag_key 0 (every channel 0..nc-1).  Channels listed more
 * than once count with their multiplicity, as in the reference's tables.
 * Out-of-range channels are rejected. */
AMBER_API int amber_cuda_set_channels(amber_cuda_ctx *ctx, int nc10, int uf_nc, const int *uf_chans);

/* ---- closed triangles and their normaliser: replaces calCR + read_rings
 * (amber_funcs.c:389-545).  rdata[4·t] = {r1, r2, r3, Num}, caller-owned,
 * room for max_tri rows; *rcount receives the full count (may exceed max_tri). */
AMBER_API int amber_cuda_calcr(amber_cuda_ctx *ctx, int max_tri, int *rcount, double *rdata);

/* Padded map side of a triangle whose largest ring is r1 (amber.c:193-197). */
AMBER_API long amber_cuda_ng1(const amber_cuda_ctx *ctx, int r1);

/* Strong scaling of one realisation over `world` processes (one per GPU): which rank computes
 * each of `ntri` closed triangles, given each triangle's largest ring r1 and that ring's map
 * side ng1 (amber_cuda_ng1).  A triangle is computed whole on one rank, so every lag array is
 * the single-process one; an r1 group (triangles sharing their maps) whose cost, ng1² per
 * triangle, is above 1/world of the total is split into ceil(cost·world/total) near-equal
 * parts, every other group stays whole, and the parts go largest first to the least-loaded
 * rank, each charged a twenty-fifth of its group's cost for the maps it builds.  Host-only (no
 * GPU, no context), integer arithmetic: every rank computes the same plan.  rank_of[ntri] out.
 * No reference counterpart (the reference runs one process per realisation). */
AMBER_API int amber_cuda_shard_plan(int ntri, const int *r1, const long *ng1, int world, int *rank_of);

/* ---- one triangle, file-ready: replaces the body of the rp loop,
 * amber.c:189-304 (v1) and amber_v2.c:189-309 (v2): fill_s2d_float ×3
 * (+ fill_s2I ×3), the OpenMP triple-product loop and the writer's scalars.
 * bldnu / numdnu: caller-owned nclen² arrays (nclen = 2·nc10 + 1), row
 * Δ2 + nc10, column Δ3 + nc10.  rdata_num is rdata[4·rp + 3] from calcr.
 * v1: *Ntri = Num/Ng1², *Num = (Ng1/N1)²·rdata_num; numdnu counts the channel
 * triplets exactly (AMBER_ERR_OVERFLOW if one exceeds INT32_MAX).
 * v2: numdnu = Σ I_r1·I_r2·I_r3 of the ring-masked sampling maps. */
AMBER_API int amber_cuda_triangle_v1(amber_cuda_ctx *ctx, int r1, int r2, int r3, double rdata_num, float *bldnu,
                           int32_t *numdnu, double *Ntri, double *Num);
AMBER_API int amber_cuda_triangle_v2(amber_cuda_ctx *ctx, int r1, int r2, int r3, float *bldnu, float *numdnu,
                           double *inv_Ng1_Ng2);

/* ---- many triangles in one call (the whole rp range of amber.c:187), FP64
 * results before the float cast of the file writer.  tri[3·t] = {r1, r2, r3}.
 * Triangles are grouped by r1 so each ring map is built once per map size.
 * bldnu[t·nclen² + …]; numdnu (int64, may be NULL); numtri (v2 mask
 * products, NULL unless want_v2).  Results are identical to calling the
 * per-triangle form in any order. */
AMBER_API int amber_cuda_triangles(amber_cuda_ctx *ctx, int ntri, const int *tri, int want_v2, double *bldnu,
                         int64_t *numdnu, double *numtri);

/* Split form for callers that time the device work alone: _run leaves the
 * results on the device, _fetch copies them to the caller's buffers. */
AMBER_API int amber_cuda_triangles_run(amber_cuda_ctx *ctx, int ntri, const int *tri, int want_v2);
AMBER_API int amber_cuda_triangles_fetch(amber_cuda_ctx *ctx, double *bldnu, int64_t *numdnu, double *numtri);

/* Lag-triple products of the last run (Σ over triangles of total_vcp·Ng1²,
 * the reference's own per-triangle work) and its device time in ms. */
AMBER_API int amber_cuda_last_run_stats(const amber_cuda_ctx *ctx, double *products, double *device_ms);
/* Device time of the last run split into map building, the contraction
 * kernel and the lag reduction (CUDA events on the launch stream), and how
 * many of the library's kernels it launched.  No reference counterpart: the
 * reference times only the whole loop (amber.c:230,285). */
/* Shape of the results the last amber_cuda_triangles_run left on the device
 * (what _fetch and amber_cuda_cyl_bs read): its triangle count (0 once the
 * channels are set again or calCR has reused the buffer), the lag width nclen
 * and whether it holds the v2 mask sums. */
AMBER_API int amber_cuda_last_run_shape(const amber_cuda_ctx *ctx, int *ntri, int *nclen, int *v2);
AMBER_API int amber_cuda_last_run_breakdown(const amber_cuda_ctx *ctx, double *ms_maps, double *ms_contract,
                                            double *ms_reduce, long *kernel_launches, long *contract_launches);

/* ---- MAPS two-point function: replaces 4_fbe/maps.c:179-210, which calls
 * cl_dnu (4_fbe/amber_funcs.c:1418-1488) for every channel pair nn1 <= nn2 of
 * the normalised grid.  On the grid the context holds (amber_cuda_load_grid*),
 * per log bin b of U = |(ia, j)|·Du in [umin, umax) (NB bins; maps.c uses 15,
 * 1 and 500): cldnu [NB][nc] = Σ over pairs with nn2 − nn1 = Δ of the pair's
 * binned mean of (Re1·Re2 + Im1·Im2)·NTiG1; numdnu [nc] = the pair count per
 * Δ; binu [NB] and num [NB] = the mean U and the sample count of the last pair
 * (nn1 = nn2 = nc − 1), which is what maps.c writes beside every row.  The
 * sums follow the reference's order and roundings, so the values are
 * bit-identical to the reference's.  numdnu, binu and num may be NULL. */
AMBER_API int amber_cuda_cl_dnu(amber_cuda_ctx *ctx, int NB, double umin, double umax, double *cldnu,
                                double *numdnu, double *binu, int *num);

/* ---- cylindrical bispectrum: the analysis stage's lag→k step on the device.
 * Replaces mabs_funcs.py get_cyl_BS (376-389: fold_quadrants 210-222, cut_nan
 * 259-260, Bdnu2Bk_fft 325-334) and, with window = 1, mfunc_winds.py
 * cylbs_win (122-136: mabs_win 88-103, blackman_nuttall 17-31), for every
 * triangle of the last amber_cuda_triangles_run at once: fold the (Δ2, Δ3)
 * quadrants, divide by mabs_norm and by the folded normaliser (denominator 0:
 * the triplet counts, as in v1 files; 1: the sampling-mask sums of a v2 run,
 * as in v2 files), cut n_cut cells at the edges, optionally window, then the
 * shifted inverse real 2D transform scaled by rc⁴·(N·dnu_mhz·rc_prime)².
 * tri_div (host, [ntri], may be NULL) divides each triangle's sums first: the v1
 * reader returns bldnu / Num (mabs_funcs.py:172-187), so pass Num for that chain.
 * out is [ntri][N][N] FP64 with N = 2·(nc10 + 1 − n_cut) − 1.  The reference
 * reads the lag arrays back from float files; here they are the FP64 sums.
 * n_cut = 0 keeps every cell (the reference's cut_nan(arr, 0) slices to an
 * empty array, so it has no output to match there). */
typedef struct amber_cuda_cylbs_params {
    int n_cut;        /* edge cells cut after folding (mabs_funcs.py n_nancut = 8) */
    int window;       /* 1: Blackman–Nuttall window, 0: none */
    int denominator;  /* 0: triplet counts, 1: sampling-mask sums (v2 run) */
    double mabs_norm; /* divisor of the folded sums (mabs_funcs.py fact·rjfac³) */
    double rc;        /* comoving distance, Mpc (mabs_funcs.py rc) */
    double rc_prime;  /* its derivative, Mpc/MHz (rc_prime) */
    double dnu_mhz;   /* channel width, MHz (dnu_mwa) */
} amber_cuda_cylbs_params;
AMBER_API int amber_cuda_cyl_bs(amber_cuda_ctx *ctx, const amber_cuda_cylbs_params *p, const double *tri_div,
                                double *out);

/* Kept for compatibility with callers of the earlier tile-width autotuner: the lag-space
 * contraction has no tile width to choose, so this returns 0 (no entries written).
 * No reference counterpart. */
AMBER_API int amber_cuda_tile_choices(const amber_cuda_ctx *ctx, int max_entries, int *nclen_class, int *tile_n,
                                      float *ms_trial_32, float *ms_trial_64);

/* ---- gridding: replaces group_loop_gridding / _without_flag
 * (3_vcg/tgefuncs.c:377-505, 511-621).  randpar[g·npar + {0,1}] = u/ν0, v/ν0
 * (float, as read from the random-groups parameters); data[g][ch][stokes][3]
 * = (re, im, wt) float; only Stokes 0 (RR) is gridded, as in the files the
 * reference writes.  Records are sorted by cell (stable, by record index) and
 * each cell is summed in record order, so the FP64 sums are bit-identical to
 * the reference's sequential loop.  Outputs are the summed grid and the
 * counts in file order (caller-owned: NN·(NN/2+1)·nc·2 and ·1 doubles). */
AMBER_API int amber_cuda_grid_vis(amber_cuda_ctx *ctx, long NN, long nc, double dU, double Umax, float nu_chan0, int flag_key,
                        long ngroups, long npar, long nstokes, const float *randpar, const float *data,
                        double *re_im_out, double *ntig_out);

/* Gridding followed by the channel collapse of the gridding stage
 * (collapse_channels, 3_vcg/tgefuncs.c:816-838, run with coll_key 1 before
 * WriteGVnAC_coll / Write_NTiG_coll, 693-724, 752-770): output channel k of a
 * cell is the sum of the gridded channels k·n_collapse .. k·n_collapse +
 * n_collapse − 1, added in that order (sums, counts and re/im alike), for
 * k < nc / n_collapse; trailing channels are dropped.  The outputs hold
 * NN·(NN/2+1)·(nc/n_collapse) cells' values (·2 for re_im).  n_collapse = 1
 * is amber_cuda_grid_vis.  The reference's gridding stage collapses by 4. */
AMBER_API int amber_cuda_grid_vis_collapsed(amber_cuda_ctx *ctx, long NN, long nc, double dU, double Umax,
                                            float nu_chan0, int flag_key, long ngroups, long npar, long nstokes,
                                            const float *randpar, const float *data, long n_collapse,
                                            double *re_im_out, double *ntig_out);

/* ---- batched requests: ensembles of realisations and estimation streams.
 * The reference estimates one realisation per process run (amber.c:21-335);
 * these calls are the batch form of amber_cuda_load_grid_packed +
 * amber_cuda_set_rings + amber_cuda_set_channels + amber_cuda_calcr +
 * amber_cuda_triangles for many realisations of uneven size at once.
 *
 * amber_cuda_enqueue copies the request's inputs (the caller may free them on
 * return) and queues it; a worker thread of the context runs it.  Requests are
 * admitted first come first served while their estimated device footprint
 * fits the context's HBM budget; the map-set batches of all admitted requests
 * run together in shared contraction launches, round by round, and a request
 * that arrives meanwhile joins at the next round.  A request's results do not
 * depend on what it shares the GPU with.  All triangles calCR closes are
 * estimated (v2 adds the sampling-mask sums).  While requests are pending,
 * make no other call on the context than these four.
 *
 * amber_cuda_wait blocks until the request is done (timeout_ms < 0: no limit;
 * AMBER_ERR_TIMEOUT when the limit passes first, the request keeps running)
 * and gives its triangle count; a failed request returns its error.
 * amber_cuda_result then copies the outputs into caller buffers and forgets
 * the request (for a failed request it returns the request's error and frees
 * what the request holds; until then a failed request keeps its copied
 * inputs): rdata [ntri][4] as amber_cuda_calcr, bldnu and numtri (v2)
 * [ntri][nclen²] FP64, numdnu [ntri][nclen²] int64, the request's latency in
 * ms from enqueue to completion and, when the request gave cylbs, the
 * cylindrical bispectra [ntri][N][N] (N = 2·(nc10 + 1 − n_cut) − 1) as
 * amber_cuda_cyl_bs makes them from the request's lag arrays, following the
 * reference's analysis of its files: denominator 0 divides each triangle by its
 * v1 file's Num (get_cyl_BS), denominator 1 (v2 requests) does not (cylbs_win).
 * Any output pointer may be NULL. */
typedef struct amber_cuda_request {
    long N1, nc;
    double Du;
    int flag_key;
    const double *re_im; /* [N1·(N1/2+1)][nc] complex as (re, im), as amber_cuda_load_grid_packed */
    const double *ntig;  /* [N1·(N1/2+1)][nc] sampling counts */
    int Nr;
    const double *ULow, *UHigh;
    int nc10;
    int uf_nc;            /* unflagged channel list when flag_key == 1 */
    const int *uf_chans;
    int want_v2;
    const amber_cuda_cylbs_params *cylbs; /* NULL, or: also the cylindrical bispectra (copied on enqueue) */
    int inputs_on_device; /* 1: re_im and ntig are device pointers on the context's device, read in place
                             when the request is admitted (keep them unchanged until it is done); 0: host
                             memory, copied on enqueue */
} amber_cuda_request;

typedef struct amber_cuda_engine_info {
    long requests_done;
    long rounds;               /* scheduling rounds run */
    long contraction_launches; /* contraction-kernel launches over all rounds */
    long max_active;           /* most requests admitted at once */
    long queued, active;       /* now */
    size_t peak_bytes;         /* most footprint admitted at once */
    size_t budget_bytes;       /* the engine's share of the context budget */
    double products;           /* lag-triple products of the finished requests */
    double busy_ms;            /* wall time spent in rounds, split into: */
    double setup_ms;           /*   cube upload, rings, channels and calCR of newly admitted requests */
    double maps_ms;            /*   ring-map batches */
    double contract_ms;        /*   contractions and lag reductions */
    double finish_ms;          /*   results back to the host, child contexts freed */
    long kernel_launches;      /* library kernels launched by the rounds (maps, contractions, reductions) */
    double contract_kernel_ms; /* device time of the contraction kernels (CUDA events on the launch stream) */
} amber_cuda_engine_info;

AMBER_API int amber_cuda_enqueue(amber_cuda_ctx *ctx, const amber_cuda_request *req, int64_t *ticket);
AMBER_API int amber_cuda_wait(amber_cuda_ctx *ctx, int64_t ticket, int timeout_ms, int *ntri);
AMBER_API int amber_cuda_result(amber_cuda_ctx *ctx, int64_t ticket, int max_tri, double *rdata, double *bldnu,
                                int64_t *numdnu, double *numtri, double *latency_ms, double *cyl_bs);
AMBER_API int amber_cuda_engine_stats(amber_cuda_ctx *ctx, amber_cuda_engine_info *info);

/* ---- allocation-free FP64 lag contraction of one triangle.  No counterpart
 * in the reference: it exists for callers that own every device allocation
 * themselves — a process that reserves its HBM budget at start-up, or an
 * application whose own caching allocator must remain the only one — and so
 * cannot let a library call cudaMalloc.  The caller passes device pointers:
 * the three ring-map sets m1, m2, m3 of the triangle (FP64 [nc][kp], the first
 * k = Ng1² entries of each row used, as the reference's fill_s2d builds them)
 * and the output lag array lag (FP64 [nclen²], nclen = 2·nc10+1, row Δ2+nc10,
 * column Δ3+nc10).  weight is a HOST array of nc channel multiplicities
 * (1 for every channel when the data are unflagged, the count of each channel
 * in uf_chans otherwise).  The result equals the plain FP64 path
 * (AMBER_PREC_FP64) of the context-based calls to FP64 rounding.
 * Scratch: one 8 MiB file-scope device array (partial lag tiles + channel
 * tables) that every GPU which loads the library holds until the process
 * exits; nc ≤ 4096 and nclen² ≤ 1044480 (nc10 ≤ 510); larger sizes are
 * rejected with AMBER_ERR_ARG.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress, with that device current), so
 * make that first call before any stream capture; the address is looked up
 * again when the device's context has changed (after a cudaDeviceReset).
 * Each call uploads its channel tables from host memory when it is made, so a
 * stream that is being captured is refused with AMBER_ERR_ARG.  Every call
 * shares the array: calls that overlap on the GPU (different streams, or host
 * threads) race.  Work is enqueued on `stream` (a cudaStream_t, NULL for the default
 * stream); the caller synchronises.  err_msg (may be NULL) receives a
 * message on failure. */
AMBER_API int amber_cuda_contract_fp64_noalloc(const double *m1, const double *m2, const double *m3, long nc,
                                               long k, long kp, int nc10, const int *weight, double *lag,
                                               void *stream, char *err_msg, size_t err_len);

#ifdef __cplusplus
}
#endif
#endif
