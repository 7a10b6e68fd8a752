/*
 * necg.h -- C ABI of the B200 engine for the NECG energy-and-gradient path.
 *
 * Drop-in boundary for the reference Python package
 * (MauricioCafiero/NBO_CorrelatedGaussians, directory python/).  Each entry
 * point names the reference function it replaces.  All pointers named *_dev are
 * CUDA device pointers, *_host are host pointers; every array is FP64,
 * C-contiguous.  `stream` is a cudaStream_t passed as void* (NULL = legacy
 * default stream).  Every function returns an NECG_* status code and never
 * throws or aborts.
 *
 * Problem layout (the state python/read_input.py:16-157 loads into
 * python/shared.py):
 *   n      particles in internal coordinates (shared.ne), 1..6
 *   nst    symmetry terms
 *   K      basis functions (shared.M)
 *   mass   n*n inverse-mass tensor, row-major
 *   ncv    n+1 charges, reference nucleus first
 *   scvv   nst symmetry weights, ALREADY divided by nst (read_input.py:141)
 *   sml    nst*n*n coordinate maps, sml[s*n*n + i*n + j] = shared.sml[i, j, s]
 *   sms    nst*3n*3n shift maps,    sms[s*9n*n + i*3n + j] = shared.sms[i, j, s]
 *   iv     K*blk packed parameters, blk = n(n+1)/2 + 3n: per basis function
 *          vech(L_k) column-major (python/utils.py:42-55), then s_k as x,y,z
 *          per particle (python/matel.py:59-84)
 *   x      [iv, C] of length K*blk + K (python/outprod.py:40-41)
 *   g      gradient of length K*blk + K: [GRADA, GRADC] (python/make_grad.py:90)
 */
#ifndef NECG_H
#define NECG_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
    NECG_OK = 0,
    NECG_ERR_ARG = 1,          /* bad argument (size, pointer, index) */
    NECG_ERR_NOT_PD = 2,       /* A_k + A_l' not positive definite for some pair */
    NECG_ERR_NONFINITE = 3,    /* a non-finite energy or gradient was produced */
    NECG_ERR_CUDA = 4,         /* a CUDA runtime call failed */
    NECG_ERR_ALLOC = 5,        /* device allocation failed */
    NECG_ERR_UNSUPPORTED = 6,  /* particle count outside 1..6 */
    NECG_ERR_CAPACITY = 7      /* K larger than the handle's K_max */
};

typedef struct necg_handle necg_handle;

/* Create a handle for one particle system and symmetry set; allocates the
 * device workspace for bases of up to K_max functions.  Host pointers.
 * Replaces the module state set up by python/read_input.py:78-157.
 * The workspace comes from the library's stream-ordered pool of the current
 * device (freed blocks are kept there for later handles); creation waits only
 * for the library's own stream, never for other streams' work. */
int necg_create(int n, int nst, int K_max, double efs, const double *mass_host,
                const double *ncv_host, const double *scvv_host, const double *sml_host,
                const double *sms_host, necg_handle **out);

/* Release a handle and its device workspace (back to the library's pool,
 * without synchronising the device).  No work that uses the handle may still
 * be running: synchronise the streams that used it first. */
int necg_destroy(necg_handle *h);

/* Bytes of device workspace the handle holds. */
long long necg_workspace_bytes(const necg_handle *h);

/* Ket-chunk widths of the energy tiles (>= 1) and gradient tiles (>= 4; the
 * partial buffer is sized for K_max / 4 chunks).  Set by the autotuner;
 * defaults are chosen per n. */
int necg_set_tiles(necg_handle *h, int lc_energy, int lc_grad);

/* Register-budget variant of the energy and gradient tile kernels (one warp
 * per block): the minimum number of resident warps per SM the kernel is
 * compiled for, one of 8, 12, 16, 20 (2, 3, 4, 5 warps per scheduler: up to
 * 255, 168, 128, 96 registers per thread).  The gradient kernel also has
 * 112 and 116: 12 and 16 warps per SM with its per-lane accumulators held in
 * shared memory instead of registers.  Set by the autotuner. */
int necg_set_variant(necg_handle *h, int minw_energy, int minw_grad);

/* Choice of the pair pass.  mode 0: ordered pairs, the loop structure of
 * python/make_grad.py:37-55 (every ordered pair, bra gradient only).  mode 1
 * (default when available): each (k >= l, P) term yields the bra gradient for
 * k and the ket gradient for l, halving the terms.  mode 2: as 1, fused with
 * the energy pass -- one pass over unordered pairs writes H, S and the
 * gradients of H and of S, combined once E is known (applies to necg_outprod;
 * the gradient-only entry points use mode 1).  Modes 1 and 2 need a symmetry
 * set closed under inverse (each sml and sms has its inverse in the set) and
 * n <= 5; otherwise NECG_ERR_UNSUPPORTED.  lc: kets per tile (1..64); minw: 8,
 * 12 or 16 warps per SM, and for mode 2 also 108 and 112 (8 and 12 warps with
 * the ket records re-read at each use instead of held in registers), 118 and
 * 122 (the same with each warp's ket record staged in shared memory), 208
 * (as 108, with the 8 warps of an SM in one block stepping through their terms
 * together), 218 (as 208, with the block's bra records staged in shared
 * memory), 228 (as 218, each warp's ket records staged too, the next one
 * copied while the current term runs), 248 (as 228 without the barrier after
 * every term), 258 and 268 (as 228, with warps 4-7 taking their per-term
 * barrier inside the term -- after the pair's Cholesky factor, inverse and
 * overlap for 258, after the kinetic and field terms (and, for n <= 3, the
 * Coulomb sum) for 268 -- so the two
 * warps of each scheduler run different parts of the term), 222 and 232 (218
 * and 228 with 12 warps per block; NECG_ERR_UNSUPPORTED where their shared
 * memory does not fit, n = 5).  Set by the autotuner. */
int necg_set_symmetric(necg_handle *h, int mode, int lc, int minw);

/* Fused pass (mode 2) with one-warp tiles (variants below 200): split the nst
 * symmetry terms of every tile over npc warps, 1 <= npc <= nst (1: no split,
 * the default).  A small basis has few tiles, each a long chain of LC x nst
 * terms; split, its tiles fill more of the GPU.  The splits' H and S sums go to
 * npc K x K buffers that one more kernel adds up in a fixed order.  No
 * counterpart in the reference (its loops have no such schedule).  Set by the
 * autotuner. */
int necg_set_splits(necg_handle *h, int npc);

/* One objective evaluation: python/outprod.py:20-76 outprod(x) -> (f, g),
 * including make_grad (python/make_grad.py:18-90).  Device pointers; H_dev and
 * S_dev (K*K) receive the symmetric matrices and may be NULL (workspace is used).
 * Asynchronous on `stream`; the pair status is read by necg_status().  With the
 * fused pass, a call that repeats the previous call's pointers, K and settings
 * launches the evaluation as one CUDA graph (captured on the handle's own stream
 * the second time the same call is seen); results are bitwise those of the
 * separate launches.  While `stream` is itself being captured, the kernels are
 * launched into that capture instead. */
int necg_outprod(necg_handle *h, int K, const double *x_dev, double *f_dev, double *g_dev,
                 double *H_dev, double *S_dev, void *stream);

/* Same as necg_outprod with host input and outputs: copies x to the device,
 * evaluates, copies f and g back and synchronises the stream.  Returns the
 * pair status of the evaluation. */
int necg_outprod_host(necg_handle *h, int K, const double *x_host, double *f_host,
                      double *g_host, void *stream);

/* One evaluation split across ranks (one process per GPU): the replacement of
 * the row-cyclic MPI split of source/outprod.f90:34-45 and
 * source/make_grad.f90:16-90 and its two MPI_REDUCE calls.  Each rank takes a
 * contiguous range [tile_begin, tile_end) of the fused pass's tiles (count from
 * necg_shard_tiles; same on every rank for the same handle settings):
 *   necg_shard_pairs   its tiles' H and S entries and gradient partials;
 *                      rows_dev (2K) = this shard's (H C, S C)
 *   -- the caller sums rows_dev over the ranks (all-reduce, 2K doubles) --
 *   necg_shard_grad    E, norm, GRADC from the summed rows (f_dev, g_dev);
 *                      sums_dev (part_stride(n) * K) = this shard's per-basis
 *                      gradient sums g_H - E g_S
 *   -- the caller sums sums_dev over the ranks (all-reduce) --
 *   necg_shard_finish  GRADA from the summed sums into g_dev
 * Every rank ends with the full f and g.  Needs the symmetry set closed under
 * inverse (NECG_ERR_UNSUPPORTED otherwise).  The three calls are one
 * evaluation: on one handle they must not interleave with other calls. */
int necg_shard_tiles(necg_handle *h, int K, int *ntiles);
int necg_shard_pairs(necg_handle *h, int K, const double *x_dev, int tile_begin, int tile_end,
                     double *rows_dev, void *stream);
int necg_shard_grad(necg_handle *h, int K, const double *x_dev, const double *rows_dev, int tile_begin,
                    int tile_end, double *f_dev, double *g_dev, double *sums_dev, void *stream);
int necg_shard_finish(necg_handle *h, int K, const double *x_dev, const double *sums_dev, double *g_dev,
                      void *stream);

/* Energy only: H, S (and optionally the kinetic and Coulomb parts Kin, Pot,
 * NULL to skip); when C_dev and en_dev are non-NULL, en_dev[0..1] receive
 * E = C^T H C / C^T S C and norm = 1 / C^T S C.
 * python/necg.py:36-58 (_build_matrices) and python/outprod.py:46-68. */
int necg_build_matrices(necg_handle *h, int K, const double *iv_dev, const double *C_dev,
                        double *H_dev, double *S_dev, double *Kin_dev, double *Pot_dev,
                        double *en_dev, void *stream);

/* python/make_grad.py:18-90 make_grad(eng, norm): gradient of the Rayleigh
 * quotient for given energy and normalisation, with GRADC from the supplied
 * H and S.  g_dev has K*blk + K entries. */
int necg_make_grad(necg_handle *h, int K, const double *iv_dev, const double *C_dev,
                   const double *H_dev, const double *S_dev, double eng, double norm,
                   double *g_dev, void *stream);

/* necg_make_grad with E and norm read from device memory (en_dev[0..1], as
 * written by necg_build_matrices): no host round trip, so a forward energy and
 * this backward gradient can be enqueued back to back or captured in a graph. */
int necg_make_grad_dev(necg_handle *h, int K, const double *iv_dev, const double *C_dev,
                       const double *H_dev, const double *S_dev, const double *en_dev,
                       double *g_dev, void *stream);

/* python/matel.py:28-210 matel(stf, ii, jj) for a batch of terms.
 * terms_dev: nterms * 3 ints (stf, ii, jj), 1-based.  out_dev: nterms * 4
 * doubles (ov, tk, ert, zht). */
int necg_matel(necg_handle *h, int K, const double *iv_dev, int nterms, const int *terms_dev,
               double *out_dev, void *stream);

/* python/rrms.py:21-120 rrms(stfe, stf, ii, jj, n1) for a batch of terms.
 * terms_dev: nterms * 5 ints (stfe, stf, ii, jj, n1), 1-based (n1 indexes the
 * 3n Cartesian components, particle-major).  out_dev: nterms * 2 doubles
 * (ov, st[n1] ov), the symmetry maps applied to both bra and ket. */
int necg_rrms(necg_handle *h, int K, const double *iv_dev, int nterms, const int *terms_dev,
              double *out_dev, void *stream);

/* The dipole loop of python/necg.py:200-244: for each Cartesian component m
 * (particle-major, 3n of them) comps_dev[m] = C^T Hd_m C / C^T Sd C with
 * Hd_m[j][i] = sum over (stfe, stf) of scvv[stf] scvv[stfe] rrms(stfe, stf, j,
 * i, m).tk and Sd the same sum of rrms.ov, taken over the lower triangle and
 * contracted with C on the fly (no K x K matrices).  dipole_dev (3 doubles,
 * may be NULL) receives sum_i ncv[i] comps[3 (i - 1) + c], the reference's
 * d7, d8, d9. */
int necg_dipole(necg_handle *h, int K, const double *iv_dev, const double *C_dev, double *comps_dev,
                double *dipole_dev, void *stream);

/* python/gradel.py:27-392 gradel(stf, ii, jj) for a batch of terms.
 * tgvl_dev, tgvls_dev: nterms * blk doubles (dH and dS with respect to the bra
 * block [vech(L_ii), s_ii]), doubled when ii == jj as the reference does. */
int necg_gradel(necg_handle *h, int K, const double *iv_dev, int nterms, const int *terms_dev,
                double *tgvl_dev, double *tgvls_dev, void *stream);

/* python/utils.py:78-106 f0(z) and df0(z) on an array (either output may be NULL). */
int necg_f0(const double *z_dev, int count, double *f_dev, double *df_dev, void *stream);

/* ---- batched evaluation -------------------------------------------------
 * Many independent instances (handles of any n, nst, K) evaluated in one step:
 * every per-pair phase is one persistent launch over a flattened queue of
 * (instance, tile) work items ordered by decreasing cost; the step is a fixed
 * sequence of eight kernels with fixed grids, so it can be captured once in a
 * CUDA graph and replayed for any plan.  No counterpart in the reference, which
 * evaluates one basis per process (python/outprod.py:20). */
typedef struct necg_batch necg_batch;

/* Capacity: instances per plan and tiles per queue. */
int necg_batch_create(int max_instances, int max_tiles, necg_batch **out);
int necg_batch_destroy(necg_batch *b);

/* Set the instances of the next step: for instance q, handle hs[q] with basis
 * size Ks[q] (<= its K_max), input x_dev[q] = [iv, C] and outputs g_dev[q]
 * (gradient) and f_dev[q] (energy; f_dev may be NULL).  Each handle's own tile
 * widths are used.  Uploads the plan on `stream`; the device plan buffer is
 * overwritten in stream order, so a step already enqueued on `stream` keeps
 * the plan it was launched with.  Two necg_batch objects used alternately let
 * the host plan one step while the previous one runs. */
int necg_batch_plan(necg_batch *b, int count, necg_handle *const *hs, const int *Ks,
                    const double *const *x_dev, double *const *g_dev, double *const *f_dev,
                    void *stream);

/* Launch one step of the current plan. */
int necg_batch_step(necg_batch *b, void *stream);

/* Capture the step into a CUDA graph (once; the graph reads the plan from
 * device memory, so it stays valid across necg_batch_plan calls with the same
 * capacity) and replay it. */
int necg_batch_graph(necg_batch *b, void *stream);
int necg_batch_replay(necg_batch *b, void *stream);

/* Per-instance status of the last step (synchronises `stream`); returns the
 * first non-OK code or NECG_OK. */
int necg_batch_status(necg_batch *b, int *status_out, void *stream);

/* The raw status words of the last planned step, without synchronising:
 * enqueues on `stream` a copy of 2 ints per instance (flags, first failing
 * pair; flags bit 1 = a pair not positive definite, bit 2 = non-finite) into
 * flags_host, which should be pinned and is valid once the stream reaches that
 * point.  For callers that keep several steps in flight. */
int necg_batch_status_async(necg_batch *b, int *flags_host, void *stream);

/* necg_outprod for callers that cannot allocate device memory (a host that
 * gives the GPU to its own fixed memory pool at start-up, a loop that cannot
 * afford an allocation's implicit synchronisation, a foreign-language driver
 * linking only this C ABI).  It allocates nothing: every intermediate lives in
 * one 32 MiB scratch array defined at file scope in the library, which every GPU
 * that loads the library holds until the process exits.  The caller passes the
 * problem constants as host arrays (layouts as for necg_create) and x, f, g in
 * device memory.  Synchronous: it returns the pair status of this evaluation.
 * A problem whose intermediates do not fit the 32 MiB returns
 * NECG_ERR_CAPACITY: K <= 779 for n = 5, nst = 24 (LiH); K <= 1143 for n = 3,
 * nst = 4 (H2); K <= 1247 for n = 2, nst = 2 (He).  The first call on a device looks up the array's device address and
 * must come before any stream capture on that device; the address is kept
 * for the life of the process, so no call may follow a cudaDeviceReset.  Calls
 * share the array, so calls that overlap on the GPU race; callers serialise
 * them.  No counterpart
 * in the reference: its outprod (python/outprod.py:20) allocates as NumPy does. */
int necg_outprod_noalloc(int n, int nst, int K, double efs, const double *mass_host,
                         const double *ncv_host, const double *scvv_host, const double *sml_host,
                         const double *sms_host, const double *x_dev, double *f_dev, double *g_dev,
                         void *stream);

/* Synchronise the handle's last stream and report the pair status of the most
 * recent evaluation: NECG_OK, NECG_ERR_NOT_PD or NECG_ERR_NONFINITE; *bad_pair
 * (may be NULL) receives the first failing pair as k*K + l, or -1. */
int necg_status(necg_handle *h, long long *bad_pair);

/* Phase timing: when enabled, necg_outprod records CUDA events on its stream
 * at the boundaries of its five phases -- prep (bra + ket records), energy
 * tiles, H C / S C + finalize, gradient tiles, gradient reduce.  Profiling aid
 * with no counterpart in the reference (which only prints wall-clock,
 * python/necg.py:119-123). */
int necg_profile(necg_handle *h, int enable);

/* Milliseconds of the five phases of the last profiled necg_outprod call
 * (synchronises its stream).  ms must hold 5 doubles. */
int necg_phase_ms(necg_handle *h, double *ms);

/* Measure the FP64 FMA throughput of the current device (TFLOP/s, FMA = 2)
 * with a register-only probe kernel: the denominator of the FP64 roofline.
 * Measurement aid with no counterpart in the reference. */
int necg_fp64_peak(int iters, double *tflops, void *stream);

/* Human-readable text for a status code. */
const char *necg_status_string(int code);

/* Algorithmic FP64 operation count of one (k, l, P) term (FMA = 2, add/mul = 1,
 * div/sqrt/rsqrt/exp = 1 each): which = 0 energy kernel, 1 ordered gradient
 * kernel, 2 one unordered term of the symmetric gradient pass (bra and ket
 * gradients), 3 one unordered term of the fused pass (H and S elements, bra
 * and ket gradients of H and of S); *special receives the div/sqrt/exp part. */
long long necg_term_flops(int n, int which, long long *special);

#ifdef __cplusplus
}
#endif
#endif /* NECG_H */
