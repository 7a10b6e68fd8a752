// necg_device.cuh -- device-side pieces shared by the single-instance kernels
// (necg_kernels.cu) and the batched persistent kernels (necg_batch.cu): the
// shared-memory accumulators, the status word, and the body of one tile of the
// fused pass.
#pragma once
#include <cuda_runtime.h>

#include "necg_lanes.cuh"
#include "necg_math.cuh"

namespace necg {

// Gradient accumulators of one lane in shared memory, interleaved by lane
// (field t of lane j at t * 32 + j): conflict-free, and not held in registers.
template <int N> struct SmemAcc {
    double *p;  // shared base + lane
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int t = 0; t < Part<N>::size; ++t) p[t * 32] = 0.0;
    }
    __device__ __forceinline__ double &g(int t) { return p[t * 32]; }
    __device__ __forceinline__ double &d() { return p[tri(N) * 32]; }
    __device__ __forceinline__ double &s(int t) { return p[(tri(N) + 1 + t) * 32]; }
};

// Block barrier that warps may reach from different places in the code (the
// non-aligned form of bar.sync: __syncthreads requires every thread of the
// block to execute the same barrier instruction).  Every warp of the block
// must still call it the same number of times.
__device__ __forceinline__ void cta_barrier() { asm volatile("barrier.sync 0;" ::: "memory"); }

// Copy a ket record of nd doubles (nd even: records are 16-byte multiples, at
// 16-byte aligned addresses) from global to shared memory without waiting:
// 16-byte cp.async per lane, one commit group per record.
__device__ __forceinline__ void ket_fetch(double *dst, const double *src, int nd, int lane) {
    for (int i = lane; 2 * i < nd; i += 32) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst + 2 * i);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src + 2 * i) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}
// Wait for this lane's copies and make the warp's copies visible to the warp.
__device__ __forceinline__ void ket_wait() {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncwarp();
}

// Status word: [0] bit flags, [1] first failing pair (row-major k*K + l).
__device__ __forceinline__ void flag_status(int *status, int flags, int pair) {
    if (!flags) return;
    atomicOr(status, flags);
    atomicMin(status + 1, pair);
}

// Where a part of a split tile of the lockstep pass writes instead of the
// main buffers (slot < 0: the main buffers): slot `slot` of x, fsym_tail_slot
// doubles holding its LC x 2 PS ket partials, then its LC x 64 H and S sums (H
// for the 32 bras, then S).  The address is formed where it is used, so that
// it does not hold registers through the term loop.
struct TileOut {
    double *x = nullptr;
    int slot = -1;
};

// Shared memory of one warp's fused tile: bra accumulators for H and S
// (2 * PS * 32 doubles), two ket tables of 16 rows (2 * 16 * 33) and two
// reduction rows (64).  Sized by the caller for its largest n.
struct FusedSmem {
    double *sacc, *krow, *kred;
    double *sket;  // SKET: two ket-record buffers of this warp (16-byte aligned)
};

// One tile of the fused pass over unordered pairs (k >= l): the symmetric
// gradient pass merged with the energy pass.  Each term gives the H element and
// overlap (summed over P into H_kl = H_lk and S_kl = S_lk) and the bra and ket
// gradients of h and of ov kept apart, since E is not known until finalize
// has run on the H and S this pass writes; the partial sum combines them as
// g_H - E g_S.  Tile t = (kb, lc): bras k = 32 kb + lane, kets l in
// [lc LC, lc LC + LC).  Bra partials: part_b[((t * 2 + which) * PS + f) * 32 +
// lane]; ket partials: part_k[((t * LC + l - l0) * 2 + which) * PS + f], which
// = 0 for H and 1 for S.
//
// Shared memory per warp must stay under 228 KB / 8 for 8 resident warps: the
// ket rows of two lanes are added with one shuffle before they are written,
// so each of the two ket tables has 16 rows.  The shuffles need the whole warp,
// so every lane evaluates a term: a lane without a pair (l > k, or k >= K)
// evaluates the finite pair (l, l, P) with zero weights, which adds nothing.
// VKET: ket records re-read at each use (fewer live registers).
// BSYNC: the warps of a block step through their tiles' terms together (a
// block barrier after every (l, P) term, so the warps sharing a scheduler
// execute the same stretch of code); every warp then runs LC x nst iterations,
// and an idle warp (no tile: idle = true, or l >= K) only takes the barriers.
// SBRA: the block's 32 bras of row block tl.x are staged in shared memory at
// sbra (field f of lane j at sbra[f * 32 + j]; rows past K hold row K - 1) and
// read there instead of from global memory.
// SKET: each (l, P) ket record is copied by the warp into one of its two
// buffers at sm.sket and read there; the copy of the next term's record
// (cp.async) runs while the current term is evaluated.
// [p0, p1): the symmetry terms this tile takes (p1 < 0: all nst).  A pass whose
// tiles split the terms writes each split's partials to its own slot (t is then
// the slot index) and each split's H, S sums to its own K x K buffer, or (xo)
// to the compact buffers of one part of a split tile.
// WB: write the bra partials to part_b (false: the caller reduces the warps'
// accumulators, left in sm.sacc, itself).
// SYNC (with BSYNC): 0 -- every warp takes the block barrier at the end of
// each term; 1, 2 -- warps 4-7 of the block take it inside the term instead
// (at term_fused's mid(1): after B, Bi, T and ov; mid(2): after tau and sig),
// so the two warps of each scheduler run different stretches of the body; 3 --
// no barrier per term (the warps only meet at the tile group's barriers).
template <int N, bool VKET, bool BSYNC = false, bool SBRA = false, bool SKET = false, int SYNC = 0, bool WB = true>
__device__ __forceinline__ void fsym_tile(int t, int2 tl, int LC, int K, int nst, const Consts<N> &cs,
                                          const double *__restrict__ bra, const double *__restrict__ ket,
                                          const double *__restrict__ C, const KetMap &kmap,
                                          double *__restrict__ H, double *__restrict__ S,
                                          double *__restrict__ part_b, double *__restrict__ part_k,
                                          int *status, FusedSmem sm, bool idle = false,
                                          const double *sbra = nullptr, int p0 = 0, int p1 = -1,
                                          TileOut xo = TileOut{}) {
    using KL = KetLayout<N>;
    constexpr int PS = Part<N>::size;
    static_assert(PS <= 32, "the symmetric pass needs tri(n) + 1 + 3n <= 32");
    // a barrier inside the term is taken only on the path that passes mid to
    // term_fused; anywhere else the warps' barrier counts would not match
    static_assert(SYNC == 0 || SYNC == 3 || (BSYNC && SBRA && SKET), "mid-term barriers need BSYNC, SBRA, SKET");
    const int lane = threadIdx.x & 31;
    double *krow0 = sm.krow, *krow1 = sm.krow + 16 * 33, *kred = sm.kred;
    const int k = tl.x * 32 + lane;
    const int l0 = tl.y * LC;
    const int l1 = BSYNC ? l0 + LC : min(l0 + LC, K);
    const bool kval = k < K && !idle;
    const double Ck = kval ? C[k] : 0.0;
    SmemAcc<N> accH{sm.sacc + lane}, accS{sm.sacc + PS * 32 + lane};
    accH.zero();
    accS.zero();
    // ket row output: lanes 2i and 2i+1 add their values of field f with one
    // exchange, lane 2i the H values (into row i of the H table), lane 2i+1 the
    // S values (row i of the S table)
    struct PairOut {
        double *r;
        bool odd;
        __device__ __forceinline__ double sum(double vh, double vs) const {
            const double keep = odd ? vs : vh;
            return keep + __shfl_xor_sync(0xffffffffu, odd ? vh : vs, 1);
        }
        __device__ __forceinline__ void put(int f, double vh, double vs) { r[f] = sum(vh, vs); }
        __device__ __forceinline__ void add(int f, double vh, double vs) { r[f] += sum(vh, vs); }
    } ko{((lane & 1) ? krow1 : krow0) + (lane >> 1) * 33, (lane & 1) != 0};
    bool ok = true;
    int flags = 0, bad = 0x7fffffff;  // smallest failing pair (row-major k K + l)
    // where this warp takes its per-term block barrier (BSYNC): 0 at the end of
    // the term, 1 / 2 at term_fused's mid(1) / mid(2), -1 nowhere.  Every warp
    // takes exactly one barrier per (l, P) term, or none (SYNC 3).
    const int sync_at = !BSYNC || SYNC == 3 ? -1 : SYNC == 0 || !((threadIdx.x >> 7) & 1) ? 0 : SYNC;
    struct MidSync {
        int at;
        __device__ __forceinline__ void operator()(int i) const {
            if (i == at) cta_barrier();
        }
    } mid{sync_at};
    const int pend = p1 < 0 ? nst : p1;
    // warp-uniform: ket l has work (always, without BSYNC); false from the
    // first l without work to the end of the tile
    auto has_work = [&](int l) { return !BSYNC || (!idle && l < K); };
    int cur = 0;  // SKET: the buffer that holds the current term's record
    if constexpr (SKET) {
        if (l0 < l1 && p0 < pend && has_work(l0))
            ket_fetch(sm.sket, ket + ((size_t)l0 * nst + p0) * KL::size, KL::size, lane);
    }
    for (int l = l0; l < l1; ++l) {
        const bool lok = has_work(l);
        double aH = 0.0, aS = 0.0, hsum = 0.0, ssum = 0.0;
        const bool active = kval && l <= k && lok;
        const BraRef b{bra + (active ? k : (lok ? l : 0)), (size_t)K};
        for (int P = p0; P < pend; ++P) {
            if (BSYNC && !lok) {
                if (sync_at >= 0) cta_barrier();
                continue;
            }
            const double *kr = ket + ((size_t)l * nst + P) * KL::size;
            if constexpr (SKET) {
                ket_wait();  // this term's record is in buffer cur
                int nl = l, nP = P + 1;
                if (nP >= pend) {
                    nl = l + 1;
                    nP = p0;
                }
                if (nl < l1 && has_work(nl))
                    ket_fetch(sm.sket + (cur ^ 1) * KL::size, ket + ((size_t)nl * nst + nP) * KL::size, KL::size,
                              lane);
                kr = sm.sket + cur * KL::size;
                cur ^= 1;
            }
            const double wb = active ? kr[KL::wC] : 0.0;
            const double wk = active && l < k ? 2.0 * Ck * kr[KL::winv] : 0.0;
            double h, ov;
            bool tok;
            if constexpr (SBRA && SKET)
                tok = term_fused<N, double>(BraSmem{sbra + lane}, KetSmem{kr}, cs, wb, wk, accH, accS, ko, h, ov,
                                            mid);
            else if constexpr (SBRA)
                tok = term_fused<N, double>(BraSmem{sbra + lane}, KetRefV{kr}, cs, wb, wk, accH, accS, ko, h, ov,
                                            mid);
            else if constexpr (SKET)
                tok = term_fused<N, double>(b, KetSmem{kr}, cs, wb, wk, accH, accS, ko, h, ov);
            else if constexpr (VKET)
                tok = term_fused<N, double>(b, KetRefV{kr}, cs, wb, wk, accH, accS, ko, h, ov);
            else
                tok = term_fused<N, double>(b, kr, cs, wb, wk, accH, accS, ko, h, ov);
            if (active) {
                if (!tok && ok) {  // the first pair of this lane that is not positive definite
                    ok = false;
                    bad = min(bad, k * K + l);
                }
                const double w = kr[KL::w];
                hsum += w * h;
                ssum += w * ov;
            }
            __syncwarp();
            // the 16 rows of both ket tables, summed as trees (four dependent
            // adds instead of sixteen), then mapped to l's frame together
            if (lane < PS) {
                double vh[16], vs[16];
#pragma unroll
                for (int r = 0; r < 16; ++r) {
                    vh[r] = krow0[r * 33 + lane];
                    vs[r] = krow1[r * 33 + lane];
                }
#pragma unroll
                for (int w = 8; w >= 1; w >>= 1)
#pragma unroll
                    for (int r = 0; r < w; ++r) {
                        vh[r] += vh[r + w];
                        vs[r] += vs[r + w];
                    }
                kred[lane] = vh[0];
                kred[32 + lane] = vs[0];
            }
            __syncwarp();
            if (lane < PS) {
                double mh, ms;
                ket_map_apply2(kmap, P, lane, PS, kred, kred + 32, mh, ms);
                aH += mh;
                aS += ms;
            }
            __syncwarp();
            if (BSYNC && sync_at == 0) cta_barrier();
        }
        if (BSYNC && !lok) continue;
        if (active) {
            if (!isfinite(hsum) || !isfinite(ssum)) {
                bad = min(bad, k * K + l);
                flags |= 2;
            }
            if (xo.slot >= 0) {
                double *hs = xo.x + (size_t)xo.slot * fsym_tail_slot(PS, LC) + (size_t)LC * 2 * PS;
                hs[(l - l0) * 64 + lane] = hsum;
                hs[(l - l0) * 64 + 32 + lane] = ssum;
            } else {
                H[(size_t)k * K + l] = hsum;
                H[(size_t)l * K + k] = hsum;
                S[(size_t)k * K + l] = ssum;
                S[(size_t)l * K + k] = ssum;
            }
        }
        if (lane < PS) {
            double *pk = xo.slot >= 0 ? xo.x + (size_t)xo.slot * fsym_tail_slot(PS, LC) + (size_t)(l - l0) * 2 * PS
                                      : part_k + ((size_t)t * LC + (l - l0)) * 2 * PS;
            pk[lane] = aH;
            pk[PS + lane] = aS;
        }
    }
    if (WB && kval) {
        double *pb = part_b + (size_t)t * 2 * PS * 32;
#pragma unroll
        for (int f = 0; f < 2 * PS; ++f) pb[f * 32 + lane] = sm.sacc[f * 32 + lane];
    }
    if (!ok) flags |= 1;
    flag_status(status, flags, bad);
    __syncwarp();
}

// Sum of the fused-pass partials of basis m for field f: its bra partials from
// the tiles of block kb = m / 32 (lane m % 32) and its ket partials from the
// tiles of chunk lc = m / LC in every block kb' >= that chunk; returns
// sum_H - E sum_S.  Only tiles in [t0, t1) count (a shard of the pass).  With
// the symmetry terms split npc ways, tile t's partials are slots t npc ..
// t npc + npc - 1.
template <int N>
__device__ __forceinline__ double fsym_sum_one(const int *__restrict__ tstart, int LC, int K, int f, int m,
                                               const double *__restrict__ part_b,
                                               const double *__restrict__ part_k, double E, int t0 = 0,
                                               int t1 = 0x7fffffff, int npc = 1) {
    constexpr int PS = Part<N>::size;
    const int kb = m >> 5, lane = m & 31;
    double sH = 0.0, sS = 0.0;
    const int sa = max(tstart[kb], t0) * npc, sb = min(tstart[kb + 1], t1) * npc;
    for (int t = sa; t < sb; ++t) {
        sH += part_b[(((size_t)t * 2 + 0) * PS + f) * 32 + lane];
        sS += part_b[(((size_t)t * 2 + 1) * PS + f) * 32 + lane];
    }
    const int lc = m / LC, ll = m - lc * LC;
    const int nkb = (K + 31) >> 5;
    int kb0 = lc * LC - 31;
    kb0 = kb0 > 0 ? (kb0 + 31) >> 5 : 0;
    for (int q = kb0; q < nkb; ++q) {
        const int t = tstart[q] + lc;
        if (t < t0 || t >= t1) continue;
        for (int pc = 0; pc < npc; ++pc) {
            const size_t base = ((size_t)(t * npc + pc) * LC + ll) * 2;
            sH += part_k[(base + 0) * PS + f];
            sS += part_k[(base + 1) * PS + f];
        }
    }
    return sH - E * sS;
}

}  // namespace necg
