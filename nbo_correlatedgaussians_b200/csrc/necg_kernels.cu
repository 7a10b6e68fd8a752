// necg_kernels.cu -- sm_100a FP64 kernels of the ECG energy+gradient path.
//
// One outprod evaluation (python/outprod.py:20-76 + python/make_grad.py:18-90)
// is the launch sequence
//   prep_bra    per basis k:     A_k, S_k, A_k S_k, A_k M A_k, i1, |L_k|^{3/2}
//   prep_ket    per (l, P):      A_l' = P^T A_l P, S_l' = sms s_l and derived data
//   energy      triangle tiles:  H_kl, S_kl for k >= l  (the matel loop)
//   rows        per row:         (H C)_i, (S C)_i
//   finalize    one block:       E = C^T H C / C^T S C, norm, GRADC
//   grad        square tiles:    sum over (l, P) of the bra gradient of
//                                2 C_l w_P (h - E ov)    (the gradel loop)
//   grad_reduce per basis k:     sum the tile partials, map A-space to vech(L)
// Tiles are one warp wide: lane = bra basis function k, while the ket (l, P)
// loops are warp-uniform, so ket records are read once per warp as broadcasts.
// The per-thread bodies live in necg_lanes.cuh.
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "necg_device.cuh"
#include "necg_kernels.cuh"
#include "necg_lanes.cuh"
#include "necg_math.cuh"

namespace necg {

// Ket records in device memory, read warp-uniformly.
struct DevKet {
    const double *p;
    __device__ __forceinline__ const double *at(size_t off) const { return p + off; }
};

template <int N>
__global__ void __launch_bounds__(128) prep_bra_kernel(const double *__restrict__ iv, int K,
                                                       Consts<N> cs, double *__restrict__ bra) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < K) prep_bra_one<N>(iv, K, cs, bra, k);
}

template <int N>
__global__ void __launch_bounds__(128) prep_ket_kernel(const double *__restrict__ iv,
                                                       const double *__restrict__ C, int K, int nst,
                                                       Consts<N> cs, const double *__restrict__ sml,
                                                       const double *__restrict__ sms,
                                                       const double *__restrict__ scvv,
                                                       double *__restrict__ ket,
                                                       const int *__restrict__ pinv) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id < K * nst) prep_ket_one<N>(iv, C, nst, cs, sml, sms, scvv, ket, id, pinv);
}

// Energy tiles over the lower triangle (the loop of python/outprod.py:49-54 and
// python/necg.py:43-50); tile list built by the host (energy_tile_count order).
// One warp per block; MINW = minimum resident warps per SM the kernel is
// compiled for (register budget 65536 / (32 MINW) per thread).
template <int N, int MINW>
__global__ void __launch_bounds__(32, MINW) energy_kernel(const int2 *__restrict__ tiles, int ntiles,
                                                     int LC, int K, int nst, Consts<N> cs,
                                                     const double *__restrict__ bra,
                                                     const double *__restrict__ ket,
                                                     double *__restrict__ H, double *__restrict__ S,
                                                     double *__restrict__ Kin,
                                                     double *__restrict__ Pot, int *status) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= ntiles) return;
    const int2 tl = tiles[warp];
    int k, l0, lend;
    if (!energy_lane_range(tl.x, tl.y, lane, LC, K, k, l0, lend)) return;
    int bad = 0;
    const int fl = energy_lane<N, double>(BraRef{bra + k, (size_t)K}, DevKet{ket}, k, l0, lend, K, nst,
                                          cs, H, S, Kin, Pot, bad);
    flag_status(status, fl, bad);
}

// rows[i] = (H C)_i, rows[K + i] = (S C)_i ; one warp per row
__global__ void __launch_bounds__(256) rows_kernel(const double *__restrict__ H,
                                                   const double *__restrict__ S,
                                                   const double *__restrict__ C, int K,
                                                   double *__restrict__ rows) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= K) return;
    const double *h = H + (size_t)warp * K;
    const double *s = S + (size_t)warp * K;
    double ah = 0.0, as = 0.0;
    for (int j = lane; j < K; j += 32) {
        const double c = C[j];
        ah += h[j] * c;
        as += s[j] * c;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ah += __shfl_xor_sync(0xffffffffu, ah, o);
        as += __shfl_xor_sync(0xffffffffu, as, o);
    }
    if (lane == 0) {
        rows[warp] = ah;
        rows[K + warp] = as;
    }
}

// E = C^T H C / C^T S C, norm = 1 / C^T S C (python/outprod.py:65-68) and
// GRADC = 2 norm (H - E S) C (python/make_grad.py:85) into gradc[0 .. K).
// scal = {E, norm, cHc, cSc}.  With `given`, E and norm are the caller's
// (make_grad(eng, norm) semantics).  One block of 1024 threads; fixed-order tree.
__global__ void __launch_bounds__(1024) finalize_kernel(const double *__restrict__ rows,
                                                        const double *__restrict__ C, int K,
                                                        double *__restrict__ scal,
                                                        double *__restrict__ f_out,
                                                        double *__restrict__ gradc, int *status,
                                                        int given, double eng, double gnorm,
                                                        const double *__restrict__ given_dev,
                                                        double *__restrict__ en_out) {
    __shared__ double sh[2][32];
    double ah = 0.0, as = 0.0;
    for (int i = threadIdx.x; i < K; i += blockDim.x) {
        ah += C[i] * rows[i];
        as += C[i] * rows[K + i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ah += __shfl_xor_sync(0xffffffffu, ah, o);
        as += __shfl_xor_sync(0xffffffffu, as, o);
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sh[0][w] = ah;
        sh[1][w] = as;
    }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        ah = lane < nw ? sh[0][lane] : 0.0;
        as = lane < nw ? sh[1][lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ah += __shfl_xor_sync(0xffffffffu, ah, o);
            as += __shfl_xor_sync(0xffffffffu, as, o);
        }
        if (lane == 0) {
            double E = ah / as, nrm = 1.0 / as;
            if (given == 1) {
                E = eng;
                nrm = gnorm;
            } else if (given == 2) {
                E = given_dev[0];
                nrm = given_dev[1];
            }
            scal[0] = E;
            scal[1] = nrm;
            scal[2] = ah;
            scal[3] = as;
            if (f_out) *f_out = E;
            if (en_out) {
                en_out[0] = E;
                en_out[1] = nrm;
            }
            if (!isfinite(E)) atomicOr(status, 2);
        }
    }
    __syncthreads();
    if (gradc) {
        const double E = scal[0], norm = scal[1];
        for (int i = threadIdx.x; i < K; i += blockDim.x)
            gradc[i] = 2.0 * norm * (rows[i] - E * rows[K + i]);
    }
}

// Gradient tiles over the full square of ordered pairs (the loop of
// python/make_grad.py:37-55, contracted with C on the fly as lines 61-79 do).
// Tile t = (kb, lc); lane k accumulates over l in the chunk and all P and
// writes its partial to part[(lc * Part::size + f) * K + k].
// SACC: accumulators in shared memory instead of registers.
template <int N, int MINW, bool SACC>
__global__ void __launch_bounds__(32, MINW) grad_kernel(int nkb, int nlc, int LC, int K, int nst,
                                                   Consts<N> cs, const double *__restrict__ bra,
                                                   const double *__restrict__ ket,
                                                   const double *__restrict__ scal, double lam,
                                                   double *__restrict__ part, int *status) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nkb * nlc) return;
    int k, lc, l0, l1;
    if (!grad_lane_range(warp, lane, nkb, LC, K, k, lc, l0, l1)) return;
    double *out = part + (size_t)lc * Part<N>::size * K + k;
    bool ok;
    if (SACC) {
        __shared__ double sacc[Part<N>::size * 32];
        SmemAcc<N> acc{sacc + lane};
        ok = grad_lane<N, double>(BraRef{bra + k, (size_t)K}, DevKet{ket}, l0, l1, nst, cs, lam, scal[0],
                                  out, (size_t)K, acc);
    } else {
        ok = grad_lane<N, double>(BraRef{bra + k, (size_t)K}, DevKet{ket}, l0, l1, nst, cs, lam, scal[0],
                                  out, (size_t)K);
    }
    if (!ok) flag_status(status, 1, k * K + l0);
}


// ---------------------------------------------------------------------------
// Symmetric gradient tiles: each unordered pair (k >= l) once.  Tile (kb, lc)
// of the lower-triangle tile list; lane = bra k.  For every ket (l, P) the
// lane adds the bra gradient of its term to its shared-memory accumulator and
// writes the term's ket gradient (in P's frame) to its row of a per-warp
// table; the warp then sums the table column by column, each lane maps one
// component back to l's frame (KetMap) and accumulates it over P.  Bra
// partials: part_b[(t * PS + f) * 32 + lane]; ket partials:
// part_k[(t * LC + l - l0) * PS + f].  Requires PS <= 32 (n <= 5).
template <int N, int MINW>
__global__ void __launch_bounds__(32, MINW) gsym_kernel(const int2 *__restrict__ tiles, int ntiles,
                                                   int LC, int K, int nst, Consts<N> cs,
                                                   const double *__restrict__ bra,
                                                   const double *__restrict__ ket,
                                                   const double *__restrict__ C,
                                                   const double *__restrict__ scal, KetMap kmap,
                                                   double *__restrict__ part_b,
                                                   double *__restrict__ part_k, int *status) {
    using KL = KetLayout<N>;
    constexpr int PS = Part<N>::size;
    static_assert(PS <= 32, "the symmetric pass needs tri(n) + 1 + 3n <= 32");
    __shared__ double sacc[PS * 32];
    __shared__ double krow[32 * 33];
    __shared__ double kred[32];
    const int t = blockIdx.x;
    const int lane = threadIdx.x;
    if (t >= ntiles) return;
    const int2 tl = tiles[t];
    const int k = tl.x * 32 + lane;
    const int l0 = tl.y * LC;
    const int l1 = min(l0 + LC, K);
    const bool kval = k < K;
    const double E = scal[0];
    const double Ck = kval ? C[k] : 0.0;
    SmemAcc<N> acc{sacc + lane};
    acc.zero();
    const BraRef b{bra + (kval ? k : 0), (size_t)K};
    struct RowOut {
        double *r;
        __device__ __forceinline__ void put(int f, double v) { r[f] = v; }
        __device__ __forceinline__ void add(int f, double v) { r[f] += v; }
    } ko{krow + lane * 33};
    bool ok = true;
    for (int l = l0; l < l1; ++l) {
        double accl = 0.0;
        for (int P = 0; P < nst; ++P) {
            const double *kr = ket + ((size_t)l * nst + P) * KL::size;
            if (kval && l <= k) {
                const double wk = l < k ? 2.0 * Ck * kr[KL::winv] : 0.0;
                ok = term_sym<N, double>(b, kr, cs, E, kr[KL::wC], wk, acc, ko) && ok;
            } else {
#pragma unroll
                for (int f = 0; f < PS; ++f) ko.r[f] = 0.0;
            }
            __syncwarp();
            double v = 0.0;
            if (lane < PS)
#pragma unroll 8
                for (int r = 0; r < 32; ++r) v += krow[r * 33 + lane];
            kred[lane] = v;
            __syncwarp();
            if (lane < PS) accl += ket_map_apply(kmap, P, lane, PS, kred);
            __syncwarp();
        }
        if (lane < PS) part_k[((size_t)t * LC + (l - l0)) * PS + lane] = accl;
    }
    if (kval) {
#pragma unroll
        for (int f = 0; f < PS; ++f) part_b[((size_t)t * PS + f) * 32 + lane] = sacc[f * 32 + lane];
    }
    if (!ok) flag_status(status, 1, k * K + l0);
}

// Fused pass over unordered pairs (k >= l): one warp per tile; the body is
// fsym_tile (necg_device.cuh), shared with the batched persistent kernel.
// blockIdx.y = pc splits the symmetry terms of every tile over npc warps (a
// small basis then still fills the GPU): split pc takes terms [pc PC, pc PC +
// PC), writes its partials to slot t npc + pc and its H, S sums to H, S + pc K^2
// (to be summed by hs_reduce_kernel); npc = 1 is the unsplit pass.
template <int N, int MINW, bool VKET, bool SKET>
__global__ void __launch_bounds__(32, MINW) fsym_kernel(const int2 *__restrict__ tiles, int t_begin, int t_end,
                                                   int LC, int K, int nst, int npc, Consts<N> cs,
                                                   const double *__restrict__ bra,
                                                   const double *__restrict__ ket,
                                                   const double *__restrict__ C, KetMap kmap,
                                                   double *__restrict__ H, double *__restrict__ S,
                                                   double *__restrict__ part_b,
                                                   double *__restrict__ part_k, int *status) {
    __shared__ double sacc[2 * Part<N>::size * 32];
    __shared__ double krow[2 * 16 * 33];
    __shared__ double kred[64];
    __shared__ __align__(16) double sket[SKET ? 2 * KetLayout<N>::size : 2];
    const int t = t_begin + blockIdx.x;
    if (t >= t_end) return;
    const int pc = blockIdx.y, PC = (nst + npc - 1) / npc;
    const int p0 = min(pc * PC, nst), p1 = min(p0 + PC, nst);
    const size_t off = (size_t)pc * K * K;
    fsym_tile<N, VKET, false, false, SKET>(t * npc + pc, tiles[t], LC, K, nst, cs, bra, ket, C, kmap, H + off,
                                           S + off, part_b, part_k, status, FusedSmem{sacc, krow, kred, sket},
                                           false, nullptr, p0, p1);
}

// H, S = sum over the npc splits of the fused pass (fixed order: deterministic).
__global__ void __launch_bounds__(256) hs_reduce_kernel(const double *__restrict__ Hp,
                                                        const double *__restrict__ Sp, int npc, size_t KK,
                                                        double *__restrict__ H, double *__restrict__ S) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < KK; i += (size_t)gridDim.x * blockDim.x) {
        double h = Hp[i], s = Sp[i];
        for (int pc = 1; pc < npc; ++pc) {
            h += Hp[pc * KK + i];
            s += Sp[pc * KK + i];
        }
        H[i] = h;
        S[i] = s;
    }
}

// The fused pass with W-warp blocks (W = 8 or 12), one per SM, persistent over
// a queue of tile groups: group g = row block kb and ket chunks lc0 .. lc0 + W
// - 1, one per warp.  The warps read the same 32 bras and step through their
// terms together (fsym_tile with BSYNC), so the warps sharing a scheduler run
// the same stretch of the long term body.  SBRA: the group's bras are staged in
// shared memory once for all warps; SKET: each warp stages its ket records in
// two buffers (the next term's copied while the current one is evaluated).
// SYNC: where the warps take their per-term barrier (fsym_tile).  Shared
// memory (dynamic, 16-byte aligned): per warp 2 PS 32 + 2 16 33 + 64 (+ 2 ket
// records) doubles, then the bras.
template <int N> __host__ __device__ constexpr int fsym_warp_smem(bool sket) {
    return 2 * Part<N>::size * 32 + 2 * 16 * 33 + 64 + (sket ? 2 * KetLayout<N>::size : 0);
}
template <int N> __host__ __device__ constexpr int fsym_block_smem_bytes(int warps, bool sbra, bool sket) {
    return (warps * fsym_warp_smem<N>(sket) + (sbra ? BraLayout<N>::size * 32 : 0)) * 8;
}

template <int N, bool VKET, bool SBRA, bool SKET, int WARPS, int SYNC = 0>
__global__ void __launch_bounds__(32 * WARPS, 1) fsym_block_kernel(const int2 *__restrict__ groups, int ngroups,
                                                                int *__restrict__ qcount,
                                                                const int *__restrict__ tstart, int LC, int K,
                                                                int nst, Consts<N> cs,
                                                                const double *__restrict__ bra,
                                                                const double *__restrict__ ket,
                                                                const double *__restrict__ C, KetMap kmap,
                                                                double *__restrict__ H, double *__restrict__ S,
                                                                double *__restrict__ part_b,
                                                                double *__restrict__ part_k, int *status,
                                                                double *__restrict__ xsym, int tail0) {
    extern __shared__ __align__(16) double smem[];
    __shared__ int gsh;
    constexpr int PS = Part<N>::size;
    constexpr int PER_WARP = fsym_warp_smem<N>(SKET);
    constexpr int BS = BraLayout<N>::size;
    const int w = threadIdx.x >> 5;
    double *base = smem + w * PER_WARP;
    double *sbra = smem + WARPS * PER_WARP;  // SBRA: BS x 32 doubles after the warps' areas
    const FusedSmem sm{base, base + 2 * PS * 32, base + 2 * PS * 32 + 2 * 16 * 33,
                       base + 2 * PS * 32 + 2 * 16 * 33 + 64};
    for (;;) {
        if (threadIdx.x == 0) gsh = atomicAdd(qcount, 1);
        __syncthreads();
        const int g = gsh;
        __syncthreads();  // every thread has read gsh before it changes
        if (g >= ngroups) break;
        const int2 gr = groups[g];
        const int kb = gr.x, lc = sgroup_lc0(gr) + w;
        const int last = min(kb * 32 + 31, K - 1);
        const bool idle = lc * LC > last;  // past this block's triangle: barriers only
        // a split group of the queue's tail: this unit takes symmetry terms
        // [p0, p1); parts after the first write to their own slots in xsym
        const int part = sgroup_part(gr), parts = sgroup_parts(gr);
        const int p0 = part * nst / parts, p1 = (part + 1) * nst / parts;  // balanced ranges
        TileOut xo;
        if (part > 0) {
            xo.x = xsym;
            xo.slot = (((g - tail0) / parts) * WARPS + w) * (parts - 1) + (part - 1);
        }
        if constexpr (SBRA) {  // the group's 32 bras, once for all warps
            for (int i = threadIdx.x; i < BS * 32; i += 32 * WARPS) {
                const int f = i >> 5, kk = min(kb * 32 + (i & 31), K - 1);
                sbra[i] = bra[(size_t)f * K + kk];
            }
            __syncthreads();
        }
        fsym_tile<N, VKET, true, SBRA, SKET, SYNC, false>(tstart[kb] + lc, make_int2(kb, lc), LC, K, nst, cs, bra,
                                                          ket, C, kmap, H, S, part_b, part_k, status, sm, idle,
                                                          sbra, p0, p1, xo);
        // the group's bra partials: its warps share the 32 bras, so their
        // accumulators are summed (in warp order) and written once, to the
        // slot of queue unit g
        __syncthreads();
        for (int i = threadIdx.x; i < 2 * PS * 32; i += 32 * WARPS) {
            if (kb * 32 + (i & 31) >= K) continue;
            double v = smem[i];
#pragma unroll
            for (int q = 1; q < WARPS; ++q) v += smem[q * PER_WARP + i];
            part_b[(size_t)g * 2 * PS * 32 + i] = v;
        }
        if constexpr (SBRA) __syncthreads();  // sbra is rewritten for the next group
    }
}

// The split tail of the lockstep pass: add parts 1 .. parts - 1 of each tile
// (their compact slots in xsym, in part order) into the tile's ket partials
// and H, S entries, which part 0 wrote (each part's bra partials have a queue
// slot of their own).  Block = one tile (tail group j, warp w); entries that no
// part wrote (kets past K or above the diagonal, tiles past the block's
// triangle) are left alone.
template <int N>
__global__ void __launch_bounds__(256) fsym_tail_fix_kernel(const int2 *__restrict__ groups, int tail0, int W,
                                                            int LC, int K, const int *__restrict__ tstart,
                                                            const double *__restrict__ xsym,
                                                            double *__restrict__ part_k, double *__restrict__ H,
                                                            double *__restrict__ S) {
    constexpr int PS = Part<N>::size;
    const int j = blockIdx.x / W, w = blockIdx.x - j * W;
    const int2 gr = groups[tail0 + j * sgroup_parts(groups[tail0])];
    const int parts = sgroup_parts(gr);
    const int kb = gr.x, lc = sgroup_lc0(gr) + w;
    const int last = min(kb * 32 + 31, K - 1);
    if (lc * LC > last) return;
    const int t = tstart[kb] + lc;
    const size_t XS = fsym_tail_slot(PS, LC);
    const double *x0 = xsym + (size_t)(j * W + w) * (parts - 1) * XS;
    double *pk = part_k + (size_t)t * LC * 2 * PS;
    for (int i = threadIdx.x; i < LC * 2 * PS; i += blockDim.x) {
        if (lc * LC + i / (2 * PS) >= K) continue;
        double v = pk[i];
        for (int q = 0; q < parts - 1; ++q) v += x0[q * XS + i];
        pk[i] = v;
    }
    for (int i = threadIdx.x; i < LC * 64; i += blockDim.x) {
        const int l = lc * LC + i / 64, r = i & 63, k = kb * 32 + (r & 31);
        if (k >= K || l >= K || l > k) continue;
        double *M = r < 32 ? H : S;
        double v = M[(size_t)k * K + l];
        for (int q = 0; q < parts - 1; ++q) v += x0[q * XS + (size_t)LC * 2 * PS + i];
        M[(size_t)k * K + l] = v;
        M[(size_t)l * K + k] = v;
    }
}

// Sum the fused-pass partials and combine out[f * K + m] = sum_H - E sum_S with
// E = scal[0] (written by finalize after the pass).  Block (kb, f): the 32
// bases of row block kb, field f.  Their bra partials come from every tile of
// block kb (up to K / LC of them) and their ket partials from one tile per
// later row block, so the 8 warps of the block take every 8th of each and
// their sums are combined in a fixed order.  Only tiles in [t0, t1) count (a
// shard of the pass).
template <int N>
__global__ void __launch_bounds__(256) fsym_sum_kernel(const int *__restrict__ tstart, int LC, int K,
                                                       const double *__restrict__ part_b,
                                                       const double *__restrict__ part_k,
                                                       const double *__restrict__ scal,
                                                       double *__restrict__ out, int t0, int t1, int npc,
                                                       const int2 *__restrict__ urange) {
    constexpr int PS = Part<N>::size;
    __shared__ double red[4][8][32];
    const int kb = blockIdx.x, f = blockIdx.y;
    const int lane = threadIdx.x & 31, seg = threadIdx.x >> 5;
    const int m = kb * 32 + lane;
    // bra partial slots: tile t's splits are slots t npc .. t npc + npc - 1, or
    // (urange, the lockstep pass) the queue units [urange[kb].x, urange[kb].y)
    const int ta = urange ? urange[kb].x : max(tstart[kb], t0) * npc;
    const int tb = urange ? urange[kb].y : min(tstart[kb + 1], t1) * npc;
    double sH = 0.0, sS = 0.0;
    for (int t = ta + seg; t < tb; t += 8) {
        sH += part_b[(((size_t)t * 2 + 0) * PS + f) * 32 + lane];
        sS += part_b[(((size_t)t * 2 + 1) * PS + f) * 32 + lane];
    }
    // the ket partials of basis m: tile (q, lc) of every row block q from
    // kb0 on, every 8th q per warp
    double kH = 0.0, kS = 0.0;
    if (m < K) {
        const int lc = m / LC, ll = m - lc * LC;
        const int nkb = (K + 31) >> 5;
        int kb0 = lc * LC - 31;
        kb0 = kb0 > 0 ? (kb0 + 31) >> 5 : 0;
        for (int q = kb0 + seg; q < nkb; q += 8) {
            const int t = tstart[q] + lc;
            if (t < t0 || t >= t1) continue;
            for (int pc = 0; pc < npc; ++pc) {
                const size_t base = ((size_t)(t * npc + pc) * LC + ll) * 2;
                kH += part_k[(base + 0) * PS + f];
                kS += part_k[(base + 1) * PS + f];
            }
        }
    }
    red[0][seg][lane] = sH;
    red[1][seg][lane] = sS;
    red[2][seg][lane] = kH;
    red[3][seg][lane] = kS;
    __syncthreads();
    if (seg != 0 || m >= K) return;
    // fixed order: the bra sums of the 8 warps, then their ket sums
    sH = red[0][0][lane];
    sS = red[1][0][lane];
#pragma unroll
    for (int q = 1; q < 8; ++q) {
        sH += red[0][q][lane];
        sS += red[1][q][lane];
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        sH += red[2][q][lane];
        sS += red[3][q][lane];
    }
    out[(size_t)f * K + m] = sH - scal[0] * sS;
}

// Sum the symmetric-pass partials of basis m into out[f * K + m]: its bra
// partials from the tiles of block kb = m / 32 (lane m % 32) and its ket
// partials from the tiles of chunk lc = m / LC in every block kb' >= that chunk.
template <int N>
__global__ void __launch_bounds__(256) gsym_sum_kernel(const int *__restrict__ tstart, int LC, int K,
                                                       const double *__restrict__ part_b,
                                                       const double *__restrict__ part_k,
                                                       double *__restrict__ out) {
    constexpr int PS = Part<N>::size;
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= PS * K) return;
    const int f = id / K, m = id - f * K;
    const int kb = m >> 5, lane = m & 31;
    double s = 0.0;
    for (int t = tstart[kb]; t < tstart[kb + 1]; ++t) s += part_b[((size_t)t * PS + f) * 32 + lane];
    const int lc = m / LC, ll = m - lc * LC;
    const int nkb = (K + 31) >> 5;
    int kb0 = lc * LC - 31;
    kb0 = kb0 > 0 ? (kb0 + 31) >> 5 : 0;
    for (int q = kb0; q < nkb; ++q) s += part_k[((size_t)(tstart[q] + lc) * LC + ll) * PS + f];
    out[(size_t)f * K + m] = s;
}

// Sum the gradient-tile partials over the ket chunks, in place into chunk 0:
// one thread per (field, k), coalesced along k.
__global__ void __launch_bounds__(256) grad_sum_kernel(double *__restrict__ part, int nlc, int K,
                                                       int PS) {
    const size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= (size_t)PS * K) return;
    double s = part[id];
    const size_t stride = (size_t)PS * K;
    for (int lc = 1; lc < nlc; ++lc) s += part[id + lc * stride];
    part[id] = s;
}

// Scale the summed partial of basis k by norm C_k (python/make_grad.py:61-79)
// and write GRADA block k in the reference's parameter order.
template <int N>
__global__ void __launch_bounds__(128) grad_reduce_kernel(const double *__restrict__ part, int K,
                                                          const double *__restrict__ bra,
                                                          const double *__restrict__ C,
                                                          const double *__restrict__ scal,
                                                          double *__restrict__ g, int *status) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    const double sc = scal[1] * (C ? C[k] : 1.0);
    if (!grad_reduce_one<N>(part, 1, K, bra, sc, g, k)) atomicOr(status, 2);
}

// python/rrms.py:21-120 rrms(stfe, stf, ii, jj, n1) per term: terms[5 t ..] =
// (stfe, stf, ii, jj, n1), 1-based; out[2 t] = ov, out[2 t + 1] = st[n1] ov.
template <int N>
__global__ void __launch_bounds__(128) rrms_kernel(const int *__restrict__ terms, int nterms, int K,
                                                   int nst, Consts<N> cs,
                                                   const double *__restrict__ ket,
                                                   double *__restrict__ out, int *status) {
    using KL = KetLayout<N>;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nterms) return;
    const int *q = terms + 5 * t;
    const int stfe = q[0] - 1, stf = q[1] - 1, ii = q[2] - 1, jj = q[3] - 1, n1 = q[4] - 1;
    if (stfe < 0 || stfe >= nst || stf < 0 || stf >= nst || ii < 0 || ii >= K || jj < 0 || jj >= K ||
        n1 < 0 || n1 >= 3 * N) {
        atomicOr(status, 4);
        out[2 * t] = out[2 * t + 1] = NAN;
        return;
    }
    double T[3 * N], ov;
    const bool ok = term_dipole<N, double>(ket + ((size_t)ii * nst + stfe) * KL::size,
                                           ket + ((size_t)jj * nst + stf) * KL::size, cs, T, ov);
    double tn = T[0];
#pragma unroll
    for (int m = 1; m < 3 * N; ++m)
        if (m == n1) tn = T[m];
    out[2 * t] = ov;
    out[2 * t + 1] = tn * ov;
    if (!ok) flag_status(status, 1, ii * K + jj);
}

// Dipole sums of python/necg.py:200-244 contracted with C on the fly, over the
// energy tiles (lower triangle): for every pair k >= l and every (Pe, P),
// weight (2 - delta_kl) C_k C_l scvv[Pe] scvv[P]; den += w ov and
// num[m] += w st[m] ov.  One warp per tile; the warp's sums go to
// part[t * (3N + 1) + m] (m = 0: den) in a fixed shuffle order.
template <int N>
__global__ void __launch_bounds__(32) dipole_kernel(const int2 *__restrict__ tiles, int ntiles, int LC,
                                                    int K, int nst, Consts<N> cs,
                                                    const double *__restrict__ ket,
                                                    const double *__restrict__ C,
                                                    double *__restrict__ part, int *status) {
    using KL = KetLayout<N>;
    constexpr int NM = 3 * N + 1;
    const int t = blockIdx.x;
    const int lane = threadIdx.x;
    if (t >= ntiles) return;
    const int2 tl = tiles[t];
    int k, l0, lend;
    double acc[NM];
#pragma unroll
    for (int m = 0; m < NM; ++m) acc[m] = 0.0;
    bool ok = true;
    if (energy_lane_range(tl.x, tl.y, lane, LC, K, k, l0, lend)) {
        const double Ck = C[k];
        for (int Pe = 0; Pe < nst; ++Pe) {
            const double *kb = ket + ((size_t)k * nst + Pe) * KL::size;
            const double wek = kb[KL::w] * Ck;
            for (int l = l0; l < lend; ++l) {
                const double wl = (l == k ? 1.0 : 2.0) * wek * C[l];
                for (int P = 0; P < nst; ++P) {
                    const double *kr = ket + ((size_t)l * nst + P) * KL::size;
                    double T[3 * N], ov;
                    ok = term_dipole<N, double>(kb, kr, cs, T, ov) && ok;
                    const double wo = wl * kr[KL::w] * ov;
                    acc[0] += wo;
#pragma unroll
                    for (int m = 0; m < 3 * N; ++m) acc[1 + m] += wo * T[m];
                }
            }
        }
    }
#pragma unroll
    for (int m = 0; m < NM; ++m) {
        double v = acc[m];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) part[(size_t)t * NM + m] = v;
    }
    if (!ok) flag_status(status, 1, k * K + l0);
}

// Sum the dipole tile partials in a fixed order (one block) and form
// comps[m] = num[m] / den (0 when den = 0, as python/necg.py:228) and the
// dipole d_c = sum_i ncv[i + 1] comps[3 i + c].
template <int N>
__global__ void __launch_bounds__(256) dipole_sum_kernel(const double *__restrict__ part, int ntiles,
                                                         Consts<N> cs, double *__restrict__ comps,
                                                         double *__restrict__ dip) {
    constexpr int NM = 3 * N + 1;
    __shared__ double red[NM][256];
    __shared__ double tot[NM];
    const int j = threadIdx.x;
#pragma unroll
    for (int m = 0; m < NM; ++m) {
        double s = 0.0;
        for (int t = j; t < ntiles; t += 256) s += part[(size_t)t * NM + m];
        red[m][j] = s;
    }
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (j < w)
#pragma unroll
            for (int m = 0; m < NM; ++m) red[m][j] += red[m][j + w];
        __syncthreads();
    }
    if (j < NM) tot[j] = red[j][0];
    __syncthreads();
    if (j < 3 * N) comps[j] = tot[0] != 0.0 ? tot[1 + j] / tot[0] : 0.0;
    __syncthreads();
    if (j < 3 && dip) {
        double d = 0.0;
        for (int i = 0; i < N; ++i) d += cs.q[i] * (tot[0] != 0.0 ? tot[1 + 3 * i + j] / tot[0] : 0.0);
        dip[j] = d;
    }
}

// Per-term elements for the matel / gradel API: terms[3 t .. 3 t + 2] =
// (stf, ii, jj), 1-based as in python/matel.py:28 and python/gradel.py:27.
template <int N>
__global__ void __launch_bounds__(128) matel_kernel(const int *__restrict__ terms, int nterms, int K,
                                                    int nst, Consts<N> cs,
                                                    const double *__restrict__ bra,
                                                    const double *__restrict__ ket,
                                                    double *__restrict__ out, int *status) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nterms) return;
    const int stf = terms[3 * t] - 1, ii = terms[3 * t + 1] - 1, jj = terms[3 * t + 2] - 1;
    if (stf < 0 || stf >= nst || ii < 0 || ii >= K || jj < 0 || jj >= K) {
        atomicOr(status, 4);
        for (int q = 0; q < 4; ++q) out[4 * t + q] = NAN;
        return;
    }
    const double *kr = ket + ((size_t)jj * nst + stf) * KetLayout<N>::size;
    if (!matel_one<N, double>(BraRef{bra + ii, (size_t)K}, kr, cs, out + 4 * t))
        flag_status(status, 1, ii * K + jj);
}

template <int N>
__global__ void __launch_bounds__(128) gradel_kernel(const int *__restrict__ terms, int nterms,
                                                     int K, int nst, Consts<N> cs,
                                                     const double *__restrict__ bra,
                                                     const double *__restrict__ ket,
                                                     double *__restrict__ tgvl,
                                                     double *__restrict__ tgvls, int *status) {
    constexpr int blk = tri(N) + 3 * N;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nterms) return;
    const int stf = terms[3 * t] - 1, ii = terms[3 * t + 1] - 1, jj = terms[3 * t + 2] - 1;
    if (stf < 0 || stf >= nst || ii < 0 || ii >= K || jj < 0 || jj >= K) {
        atomicOr(status, 4);
        for (int q = 0; q < blk; ++q) tgvl[(size_t)t * blk + q] = tgvls[(size_t)t * blk + q] = NAN;
        return;
    }
    const double *kr = ket + ((size_t)jj * nst + stf) * KetLayout<N>::size;
    double L[tri(N)];
#pragma unroll
    for (int q = 0; q < tri(N); ++q) L[q] = bra[(BraLayout<N>::L + q) * (size_t)K + ii];
    if (!gradel_one<N, double>(BraRef{bra + ii, (size_t)K}, kr, cs, L, ii == jj,
                               tgvl + (size_t)t * blk, tgvls + (size_t)t * blk))
        flag_status(status, 1, ii * K + jj);
}

// FP64 throughput probe: 8 independent FMA chains per thread, all in
// registers.  Used to measure the FP64 roofline denominator on the running GPU.
__global__ void __launch_bounds__(256) fp64_probe_kernel(int iters, double seed, double *sink) {
    double a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = seed + threadIdx.x * 1e-7 + j;
    const double b = 0.999999999, c = 1e-9;
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = fma(a[j], b, c);
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += a[j];
    if (s == 12345.6789) sink[blockIdx.x] = s;  // never true; keeps the chains live
}

// Boys function on an array (python/utils.py:78-106)
__global__ void f0_kernel(const double *__restrict__ z, int count, double *__restrict__ f,
                          double *__restrict__ df) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    double fs, D, ia, zo;
    boys<true>(1.0, z[i], fs, D, ia, zo);  // a = 1: fs = F0(z), D = F0'(z) / F0(z)
    if (f) f[i] = fs;
    if (df) df[i] = fs * D;
}

__global__ void reset_status_kernel(int *status) {
    status[0] = 0;
    status[1] = 0x7fffffff;
}

// ---------------------------------------------------------------------------
// Host-side launchers (one instantiation per supported particle count)
template <int N> Consts<N> make_consts(const double *mass, const double *ncv, double efs) {
    Consts<N> c;
    for (int i = 0; i < N * N; ++i) c.M[i] = mass[i];
    c.derive();
    for (int q = 1; q <= N; ++q)
        for (int p = 0; p < q; ++p) c.cv[vidx(p, q)] = 2.0 * ncv[p] * ncv[q] / NECG_SQRT_PI;
    for (int i = 0; i < N; ++i) c.q[i] = ncv[i + 1];
    c.efs = efs;
    c.sqrt8n = sqrt(pow(8.0, N));
    return c;
}

template <int N> struct Launch {
    static void prep(const LaunchArgs &a, cudaStream_t st) {
        Consts<N> cs = make_consts<N>(a.mass_h, a.ncv_h, a.efs);
        prep_bra_kernel<N><<<(a.K + 127) / 128, 128, 0, st>>>(a.iv, a.K, cs, a.bra);
        const int nk = a.K * a.nst;
        prep_ket_kernel<N><<<(nk + 127) / 128, 128, 0, st>>>(a.iv, a.C, a.K, a.nst, cs, a.sml, a.sms,
                                                             a.scvv, a.ket, a.pinv);
    }
    template <int MINW> static void energy_v(const LaunchArgs &a, cudaStream_t st) {
        Consts<N> cs = make_consts<N>(a.mass_h, a.ncv_h, a.efs);
        energy_kernel<N, MINW><<<a.ntiles, 32, 0, st>>>(a.tiles, a.ntiles, a.LC_e, a.K, a.nst, cs, a.bra,
                                                        a.ket, a.H, a.S, a.Kin, a.Pot, a.status);
    }
    static void energy(const LaunchArgs &a, cudaStream_t st) {
        switch (a.minb_e) {
        case 12: energy_v<12>(a, st); break;
        case 16: energy_v<16>(a, st); break;
        case 20: energy_v<20>(a, st); break;
        default: energy_v<8>(a, st); break;
        }
    }
    template <int MINW, bool SACC> static void grad_v(const LaunchArgs &a, cudaStream_t st) {
        Consts<N> cs = make_consts<N>(a.mass_h, a.ncv_h, a.efs);
        const int nkb = (a.K + 31) / 32, nlc = (a.K + a.LC_g - 1) / a.LC_g;
        grad_kernel<N, MINW, SACC><<<nkb * nlc, 32, 0, st>>>(nkb, nlc, a.LC_g, a.K, a.nst, cs, a.bra,
                                                             a.ket, a.scal, a.lam, a.part, a.status);
    }
    // variant codes: 8, 12, 16, 20 = warps per SM with register accumulators;
    // 112, 116 = 12, 16 warps per SM with shared-memory accumulators
    static void grad_tiles(const LaunchArgs &a, cudaStream_t st) {
        switch (a.minb_g) {
        case 12: grad_v<12, false>(a, st); break;
        case 16: grad_v<16, false>(a, st); break;
        case 20: grad_v<20, false>(a, st); break;
        case 112: grad_v<12, true>(a, st); break;
        case 116: grad_v<16, true>(a, st); break;
        default: grad_v<8, false>(a, st); break;
        }
    }
    static void grad_reduce(const LaunchArgs &a, cudaStream_t st) {
        const int nlc = (a.K + a.LC_g - 1) / a.LC_g;
        constexpr int PS = Part<N>::size;
        const size_t nthr = (size_t)PS * a.K;
        if (nlc > 1) grad_sum_kernel<<<(unsigned)((nthr + 255) / 256), 256, 0, st>>>(a.part, nlc, a.K, PS);
        grad_reduce_kernel<N><<<(a.K + 127) / 128, 128, 0, st>>>(a.part, a.K, a.bra, a.C, a.scal, a.g,
                                                                  a.status);
    }
    template <int MINW> static void gsym_v(const LaunchArgs &a, cudaStream_t st) {
        if constexpr (Part<N>::size <= 32) {
            Consts<N> cs = make_consts<N>(a.mass_h, a.ncv_h, a.efs);
            gsym_kernel<N, MINW><<<a.nstiles, 32, 0, st>>>(a.stiles, a.nstiles, a.LC_s, a.K, a.nst, cs, a.bra,
                                                           a.ket, a.C, a.scal, a.kmap, a.psym,
                                                           a.psym + (size_t)a.nstiles * Part<N>::size * 32,
                                                           a.status);
        }
    }
    static void gsym_tiles(const LaunchArgs &a, cudaStream_t st) {
        switch (a.minb_s) {
        case 12: gsym_v<12>(a, st); break;
        case 16: gsym_v<16>(a, st); break;
        default: gsym_v<8>(a, st); break;
        }
    }
    static void gsym_reduce(const LaunchArgs &a, cudaStream_t st) {
        if constexpr (Part<N>::size <= 32) {
            constexpr int PS = Part<N>::size;
            gsym_sum_kernel<N><<<(PS * a.K + 255) / 256, 256, 0, st>>>(
                a.stile_start, a.LC_s, a.K, a.psym, a.psym + (size_t)a.nstiles * PS * 32, a.part);
            grad_reduce_kernel<N><<<(a.K + 127) / 128, 128, 0, st>>>(a.part, a.K, a.bra, a.C, a.scal, a.g,
                                                                      a.status);
        }
    }
    template <int MINW, bool VKET, bool SKET = false> static void fsym_v(const LaunchArgs &a, cudaStream_t st) {
        if constexpr (Part<N>::size <= 32) {
            Consts<N> cs = make_consts<N>(a.mass_h, a.ncv_h, a.efs);
            const int t0 = a.st_end > 0 ? a.st_begin : 0, t1 = a.st_end > 0 ? a.st_end : a.nstiles;
            if (t1 <= t0) return;
            const int npc = a.npc > 1 ? a.npc : 1;
            fsym_kernel<N, MINW, VKET, SKET><<<dim3(t1 - t0, npc), 32, 0, st>>>(
                a.stiles, t0, t1, a.LC_s, a.K, a.nst, npc, cs, a.bra, a.ket, a.C, a.kmap, npc > 1 ? a.Hp : a.H,
                npc > 1 ? a.Sp : a.S, a.psym, a.psym + (size_t)a.nstiles * npc * 2 * Part<N>::size * 32, a.status);
        }
    }
    template <bool SBRA, bool SKET, int WARPS, int SYNC = 0>
    static void fsym_block(const LaunchArgs &a, cudaStream_t st) {
        if constexpr (Part<N>::size <= 32) {
            constexpr int smem = fsym_block_smem_bytes<N>(WARPS, SBRA, SKET);
            if constexpr (smem <= 232448) {
                auto kern = fsym_block_kernel<N, true, SBRA, SKET, WARPS, SYNC>;
                int dev = 0, sms = 148;
                cudaGetDevice(&dev);
                // the shared-memory opt-in is per device: once per instantiation and device
                static bool attr[64] = {};
                if (dev < 0 || dev >= 64 || !attr[dev]) {
                    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
                    if (dev >= 0 && dev < 64) attr[dev] = true;
                }
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
                Consts<N> cs = make_consts<N>(a.mass_h, a.ncv_h, a.efs);
                cudaMemsetAsync(a.qcount, 0, sizeof(int), st);
                const int grid = a.nsgroups < sms ? a.nsgroups : sms;
                if (grid < 1) return;
                kern<<<grid, 32 * WARPS, smem, st>>>(a.sgroups, a.nsgroups, a.qcount, a.stile_start, a.LC_s, a.K,
                                                     a.nst, cs, a.bra, a.ket, a.C, a.kmap, a.H, a.S, a.psym,
                                                     a.psym + (size_t)a.nstiles * 2 * Part<N>::size * 32, a.status,
                                                     a.xsym, a.sg_tail0);
            }
        }
    }
    static void fsym_tiles(const LaunchArgs &a, cudaStream_t st) {
        if (a.minb_s >= 200 && a.st_end == 0 && a.sgroups && a.qcount) {
            switch (a.minb_s) {  // 2xy: lockstep blocks; see fused_variant_ok
            case 218: fsym_block<true, false, 8>(a, st); break;
            case 228: fsym_block<true, true, 8>(a, st); break;
            case 248: fsym_block<true, true, 8, 3>(a, st); break;
            case 258: fsym_block<true, true, 8, 1>(a, st); break;
            case 268: fsym_block<true, true, 8, 2>(a, st); break;
            case 222: fsym_block<true, false, 12>(a, st); break;
            case 232: fsym_block<true, true, 12>(a, st); break;
            default: fsym_block<false, false, 8>(a, st); break;
            }
            return;
        }
        switch (a.minb_s) {  // 100 + w: ket records read at the point of use
        case 12: fsym_v<12, false>(a, st); break;
        case 16: fsym_v<16, false>(a, st); break;
        case 108: fsym_v<8, true>(a, st); break;
        case 112: fsym_v<12, true>(a, st); break;
        case 118: fsym_v<8, true, true>(a, st); break;
        case 122: fsym_v<12, true, true>(a, st); break;
        default: fsym_v<8, false>(a, st); break;
        }
    }
    static void fsym_tail(const LaunchArgs &a, cudaStream_t st) {
        if constexpr (Part<N>::size <= 32) {
            const int W = fused_block_warps(a.minb_s);
            fsym_tail_fix_kernel<N><<<a.sg_ntail * W, 256, 0, st>>>(
                a.sgroups, a.sg_tail0, W, a.LC_s, a.K, a.stile_start, a.xsym,
                a.psym + (size_t)a.nstiles * 2 * Part<N>::size * 32, a.H, a.S);
        }
    }
    static void fsym_reduce(const LaunchArgs &a, cudaStream_t st) {
        if constexpr (Part<N>::size <= 32) {
            constexpr int PS = Part<N>::size;
            const int t0 = a.st_end > 0 ? a.st_begin : 0, t1 = a.st_end > 0 ? a.st_end : a.nstiles;
            const int npc = a.npc > 1 && a.minb_s < 200 ? a.npc : 1;
            // the lockstep pass over the whole tile list writes its bra partials
            // per queue unit (the unit ranges of each row block in urange)
            const bool lockstep = a.minb_s >= 200 && a.st_end == 0 && a.sgroups && a.urange;
            fsym_sum_kernel<N><<<dim3((a.K + 31) / 32, PS), 256, 0, st>>>(
                a.stile_start, a.LC_s, a.K, a.psym, a.psym + (size_t)a.nstiles * npc * 2 * PS * 32, a.scal,
                a.sums ? a.sums : a.part, t0, t1, npc, lockstep ? a.urange : nullptr);
            if (!a.sums)
                grad_reduce_kernel<N><<<(a.K + 127) / 128, 128, 0, st>>>(a.part, a.K, a.bra, a.C, a.scal, a.g,
                                                                          a.status);
        }
    }
    static void rrms(const LaunchArgs &a, const int *terms, int nterms, double *out, cudaStream_t st) {
        Consts<N> cs = make_consts<N>(a.mass_h, a.ncv_h, a.efs);
        rrms_kernel<N><<<(nterms + 127) / 128, 128, 0, st>>>(terms, nterms, a.K, a.nst, cs, a.ket, out,
                                                             a.status);
    }
    static void dipole(const LaunchArgs &a, double *part, double *comps, double *dip, cudaStream_t st) {
        Consts<N> cs = make_consts<N>(a.mass_h, a.ncv_h, a.efs);
        dipole_kernel<N><<<a.ntiles, 32, 0, st>>>(a.tiles, a.ntiles, a.LC_e, a.K, a.nst, cs, a.ket, a.C, part,
                                                  a.status);
        dipole_sum_kernel<N><<<1, 256, 0, st>>>(part, a.ntiles, cs, comps, dip);
    }
    static void reduce_sums(const LaunchArgs &a, const double *sums, cudaStream_t st) {
        grad_reduce_kernel<N><<<(a.K + 127) / 128, 128, 0, st>>>(sums, a.K, a.bra, a.C, a.scal, a.g, a.status);
    }
    static void matel(const LaunchArgs &a, const int *terms, int nterms, double *out,
                      cudaStream_t st) {
        Consts<N> cs = make_consts<N>(a.mass_h, a.ncv_h, a.efs);
        matel_kernel<N><<<(nterms + 127) / 128, 128, 0, st>>>(terms, nterms, a.K, a.nst, cs, a.bra,
                                                              a.ket, out, a.status);
    }
    static void gradel(const LaunchArgs &a, const int *terms, int nterms, double *tg, double *tgs,
                       cudaStream_t st) {
        Consts<N> cs = make_consts<N>(a.mass_h, a.ncv_h, a.efs);
        gradel_kernel<N><<<(nterms + 127) / 128, 128, 0, st>>>(terms, nterms, a.K, a.nst, cs, a.bra,
                                                               a.ket, tg, tgs, a.status);
    }
};

#define NECG_DISPATCH(n, call)      \
    switch (n) {                    \
    case 1: Launch<1>::call; break; \
    case 2: Launch<2>::call; break; \
    case 3: Launch<3>::call; break; \
    case 4: Launch<4>::call; break; \
    case 5: Launch<5>::call; break; \
    case 6: Launch<6>::call; break; \
    default: return -1;             \
    }

int launch_prep(const LaunchArgs &a, cudaStream_t st) {
    NECG_DISPATCH(a.n, prep(a, st));
    return 0;
}
int launch_energy(const LaunchArgs &a, cudaStream_t st) {
    NECG_DISPATCH(a.n, energy(a, st));
    return 0;
}
int launch_grad_tiles(const LaunchArgs &a, cudaStream_t st) {
    NECG_DISPATCH(a.n, grad_tiles(a, st));
    return 0;
}
int launch_grad_reduce(const LaunchArgs &a, cudaStream_t st) {
    NECG_DISPATCH(a.n, grad_reduce(a, st));
    return 0;
}
int launch_grad(const LaunchArgs &a, cudaStream_t st) {
    if (launch_grad_tiles(a, st)) return -1;
    return launch_grad_reduce(a, st);
}
int launch_gsym(const LaunchArgs &a, cudaStream_t st) {
    if (a.n > 5) return -1;
    NECG_DISPATCH(a.n, gsym_tiles(a, st));
    return 0;
}
int launch_gsym_reduce(const LaunchArgs &a, cudaStream_t st) {
    if (a.n > 5) return -1;
    NECG_DISPATCH(a.n, gsym_reduce(a, st));
    return 0;
}
int fused_block_warps(int variant) { return variant == 222 || variant == 232 ? 12 : 8; }
bool fused_variant_ok(int n, int variant) {
    if (variant < 200) return true;
    if (n < 1 || n > 5) return false;
    const bool sbra = variant != 208,
               sket = variant == 228 || variant == 232 || variant == 248 || variant == 258 || variant == 268;
    const int warps = fused_block_warps(variant);
    int bytes = 0;
    switch (n) {
    case 1: bytes = fsym_block_smem_bytes<1>(warps, sbra, sket); break;
    case 2: bytes = fsym_block_smem_bytes<2>(warps, sbra, sket); break;
    case 3: bytes = fsym_block_smem_bytes<3>(warps, sbra, sket); break;
    case 4: bytes = fsym_block_smem_bytes<4>(warps, sbra, sket); break;
    default: bytes = fsym_block_smem_bytes<5>(warps, sbra, sket); break;
    }
    return bytes <= 232448;
}
int launch_fsym(const LaunchArgs &a, cudaStream_t st) {
    if (a.n > 5) return -1;
    // every buffer the pass writes must be set (no launch on a null pointer)
    if (!a.H || !a.S || !a.psym || !a.stiles || !a.bra || !a.ket || !a.C || !a.status) return -1;
    NECG_DISPATCH(a.n, fsym_tiles(a, st));
    return 0;
}
int launch_fsym_tail(const LaunchArgs &a, cudaStream_t st) {
    // only the lockstep pass over the whole tile list splits its tail
    if (a.minb_s < 200 || a.st_end > 0 || a.sg_ntail <= 0 || a.sg_parts < 2) return 0;
    if (a.n > 5 || !a.sgroups || !a.xsym || !a.psym || !a.H || !a.S || !a.stile_start) return -1;
    NECG_DISPATCH(a.n, fsym_tail(a, st));
    return 0;
}
int launch_fsym_reduce(const LaunchArgs &a, cudaStream_t st) {
    if (a.n > 5) return -1;
    if (!a.stile_start || !a.psym || !a.scal || (!a.sums && (!a.part || !a.bra || !a.C || !a.g))) return -1;
    NECG_DISPATCH(a.n, fsym_reduce(a, st));
    return 0;
}
int launch_hs_reduce(const LaunchArgs &a, cudaStream_t st) {
    if (a.npc <= 1) return 0;
    if (!a.Hp || !a.Sp || !a.H || !a.S) return -1;
    const size_t KK = (size_t)a.K * a.K;
    const size_t blocks = (KK + 255) / 256 < 4096 ? (KK + 255) / 256 : 4096;
    hs_reduce_kernel<<<(int)blocks, 256, 0, st>>>(a.Hp, a.Sp, a.npc, KK, a.H, a.S);
    return 0;
}
int launch_reduce_sums(const LaunchArgs &a, const double *sums, cudaStream_t st) {
    if (!sums || !a.bra || !a.C || !a.scal || !a.g || !a.status) return -1;
    NECG_DISPATCH(a.n, reduce_sums(a, sums, st));
    return 0;
}
int launch_rrms(const LaunchArgs &a, const int *terms, int nterms, double *out, cudaStream_t st) {
    NECG_DISPATCH(a.n, rrms(a, terms, nterms, out, st));
    return 0;
}
int launch_dipole(const LaunchArgs &a, double *part, double *comps, double *dip, cudaStream_t st) {
    NECG_DISPATCH(a.n, dipole(a, part, comps, dip, st));
    return 0;
}
int launch_matel(const LaunchArgs &a, const int *terms, int nterms, double *out, cudaStream_t st) {
    NECG_DISPATCH(a.n, matel(a, terms, nterms, out, st));
    return 0;
}
int launch_gradel(const LaunchArgs &a, const int *terms, int nterms, double *tg, double *tgs,
                  cudaStream_t st) {
    NECG_DISPATCH(a.n, gradel(a, terms, nterms, tg, tgs, st));
    return 0;
}
void launch_rows_finalize(const LaunchArgs &a, double *f_out, double *gradc, int given, double eng,
                          double norm, cudaStream_t st, const double *given_dev, double *en_out) {
    rows_kernel<<<(a.K * 32 + 255) / 256, 256, 0, st>>>(a.H, a.S, a.C, a.K, a.rows);
    finalize_kernel<<<1, 1024, 0, st>>>(a.rows, a.C, a.K, a.scal, f_out, gradc, a.status, given, eng,
                                        norm, given_dev, en_out);
}
int launch_rows(const LaunchArgs &a, double *rows, cudaStream_t st) {
    if (!a.H || !a.S || !a.C || !rows) return -1;
    rows_kernel<<<(a.K * 32 + 255) / 256, 256, 0, st>>>(a.H, a.S, a.C, a.K, rows);
    return 0;
}
void launch_finalize(const LaunchArgs &a, const double *rows, double *f_out, double *gradc, cudaStream_t st) {
    finalize_kernel<<<1, 1024, 0, st>>>(rows, a.C, a.K, a.scal, f_out, gradc, a.status, 0, 0.0, 0.0, nullptr,
                                        nullptr);
}
void launch_reset_status(int *status, cudaStream_t st) { reset_status_kernel<<<1, 1, 0, st>>>(status); }
void launch_fp64_probe(int blocks, int iters, double *sink, cudaStream_t st) {
    fp64_probe_kernel<<<blocks, 256, 0, st>>>(iters, 1.0, sink);
}
void launch_f0(const double *z, int count, double *f, double *df, cudaStream_t st) {
    f0_kernel<<<(count + 255) / 256, 256, 0, st>>>(z, count, f, df);
}

int ket_record_size(int n) {
    switch (n) {
    case 1: return KetLayout<1>::size;
    case 2: return KetLayout<2>::size;
    case 3: return KetLayout<3>::size;
    case 4: return KetLayout<4>::size;
    case 5: return KetLayout<5>::size;
    case 6: return KetLayout<6>::size;
    default: return 0;
    }
}
int bra_record_size(int n) {
    switch (n) {
    case 1: return BraLayout<1>::size;
    case 2: return BraLayout<2>::size;
    case 3: return BraLayout<3>::size;
    case 4: return BraLayout<4>::size;
    case 5: return BraLayout<5>::size;
    case 6: return BraLayout<6>::size;
    default: return 0;
    }
}
int part_stride(int n) { return n >= 1 && n <= 6 ? tri(n) + 1 + 3 * n : 0; }

}  // namespace necg
