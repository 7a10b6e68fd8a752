// necg_batch.cu -- many independent instances (different n, nst, K) in one
// energy+gradient step: the same math as the single-instance path, with every
// per-pair kernel a persistent launch that pulls (instance, tile) work items
// from a flattened queue.
//
// Step sequence (fixed grids, so one captured CUDA graph per mode serves any
// plan).  Fused mode (every instance's symmetry set closed under inverse):
//   reset        queue heads and per-instance status words
//   prep         grid-stride over all (instance, k) bra and (instance, l, P) ket records
//   fused        persistent warps over the fused tile queue (all instances): H, S
//                and the H and S gradient partials in one pass over unordered pairs
//   rows         grid-stride warps over all (instance, row): (H C)_i, (S C)_i
//   finalize     block per instance: E, norm, GRADC
//   fsum         grid-stride over all (instance, field, k): g_H - E g_S
//   reduce       grid-stride over all (instance, k): GRADA blocks
// Ordered mode (any other set): energy tiles over the triangle and gradient
// tiles over ordered pairs in place of fused, and a plain partial sum.
// The plan (instance table, prefix sums, tile queues ordered by decreasing
// cost) is built on the host and copied to device buffers before the step.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "necg_device.cuh"
#include "necg_handle.h"
#include "necg_lanes.cuh"
#include "necg_math.cuh"
#include "necg_trace.h"

namespace necg {

constexpr int kMaxN = 5;  // batched path: n <= 5 (He, H2, LiH and the like)
constexpr int kConstsDoubles = 128;  // >= sizeof(Consts<6>) / 8

struct InstDesc {
    int n, K, nst, lc_e, lc_g, nlc;
    int lc_s, nstiles;
    const double *iv, *C;
    double *bra, *ket, *part, *H, *S, *rows, *scal, *g, *f;
    const double *sml, *sms, *scvv;
    int *status;
    // fused mode
    const int *pinv, *stile_start;
    const int2 *stiles;  // the instance's fused tile list (kb, lc), on the device
    const int2 *bgroups; // groups of 8 consecutive chunks of one row block (kb, first lc)
    int nbgroups;
    int npc;             // one-warp fused kernel: symmetry terms split npc ways per tile
    double *psym;
    double *Hp, *Sp;     // npc > 1: the splits' H, S sums (npc K x K each)
    KetMap kmap;
    double cs[kConstsDoubles];
};

struct PlanHdr {
    int ninst, ne, ng;
    int qe, qg;  // persistent queue heads
    int nf, qf;  // fused queue: tile groups (lockstep kernel) or tiles (one-warp kernel)
    int fine;    // 1: the one-warp fused kernel (few groups for the SMs)
};

// plan buffer layout: [PlanHdr][InstDesc x cap][prefix arrays][tiles]
struct PlanPtrs {
    PlanHdr *hdr;
    InstDesc *inst;
    int *pref_bra;  // cumulative K            (ninst + 1)
    int *pref_ket;  // cumulative K * nst      (ninst + 1)
    int *pref_sum;  // cumulative PS * K       (ninst + 1)
    int *pref_ft;   // cumulative fused tile groups, or tiles when fine (ninst + 1), over `order`
    int *order;     // instances by decreasing tile cost (fused queue order)
    int4 *etiles;   // (inst, kb, lc, 0); fused mode: (inst, kb, lc, tile index in the instance)
    int4 *gtiles;
    int *status_all;  // device only: every instance's status word pair, gathered after the step
};

__device__ __forceinline__ int find_inst(const int *pref, int ninst, int i) {
    int lo = 0, hi = ninst;  // pref[lo] <= i < pref[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pref[mid] <= i) lo = mid;
        else hi = mid;
    }
    return lo;
}

template <int N> __device__ __forceinline__ const Consts<N> &consts_of(const InstDesc &d) {
    return *reinterpret_cast<const Consts<N> *>(d.cs);
}

__device__ __forceinline__ void flag_inst(int *status, int flags, int pair) {
    if (!flags) return;
    atomicOr(status, flags);
    atomicMin(status + 1, pair);
}

#define BATCH_SWITCH(n, body)                          \
    switch (n) {                                       \
    case 1: { constexpr int N = 1; body; } break;      \
    case 2: { constexpr int N = 2; body; } break;      \
    case 3: { constexpr int N = 3; body; } break;      \
    case 4: { constexpr int N = 4; body; } break;      \
    case 5: { constexpr int N = 5; body; } break;      \
    default: break;                                    \
    }

__global__ void batch_reset_kernel(PlanPtrs p) {
    const PlanHdr h = *p.hdr;
    for (int i = threadIdx.x; i < h.ninst; i += blockDim.x) {
        p.inst[i].status[0] = 0;
        p.inst[i].status[1] = 0x7fffffff;
    }
    if (threadIdx.x == 0) {
        p.hdr->qe = 0;
        p.hdr->qg = 0;
        p.hdr->qf = 0;
    }
}

__global__ void __launch_bounds__(128) batch_prep_kernel(PlanPtrs p) {
    const int ninst = p.hdr->ninst;
    const int nb = p.pref_bra[ninst], nk = p.pref_ket[ninst];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb + nk; i += gridDim.x * blockDim.x) {
        if (i < nb) {
            const int q = find_inst(p.pref_bra, ninst, i);
            const InstDesc &d = p.inst[q];
            const int k = i - p.pref_bra[q];
            BATCH_SWITCH(d.n, prep_bra_one<N>(d.iv, d.K, consts_of<N>(d), d.bra, k));
        } else {
            const int j = i - nb;
            const int q = find_inst(p.pref_ket, ninst, j);
            const InstDesc &d = p.inst[q];
            const int id = j - p.pref_ket[q];
            BATCH_SWITCH(d.n, prep_ket_one<N>(d.iv, d.C, d.nst, consts_of<N>(d), d.sml, d.sms, d.scvv,
                                             d.ket, id, d.pinv));
        }
    }
}

struct DevKetB {
    const double *p;
    __device__ __forceinline__ const double *at(size_t off) const { return p + off; }
};

__global__ void __launch_bounds__(32) batch_energy_kernel(PlanPtrs p) {
    const int lane = threadIdx.x & 31;
    const int ne = p.hdr->ne;
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(&p.hdr->qe, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= ne) break;
        const int4 e = p.etiles[t];
        const InstDesc &d = p.inst[e.x];
        int k, l0, lend;
        if (energy_lane_range(e.y, e.z, lane, d.lc_e, d.K, k, l0, lend)) {
            int bad = 0, fl = 0;
            BATCH_SWITCH(d.n, fl = (energy_lane<N, double>(BraRef{d.bra + k, (size_t)d.K}, DevKetB{d.ket}, k,
                                                           l0, lend, d.K, d.nst, consts_of<N>(d), d.H,
                                                           d.S, nullptr, nullptr, bad)));
            flag_inst(d.status, fl, bad);
        }
    }
}

// Fused tiles of every instance, one warp per tile (the plan's choice when its
// groups are too few to fill the SMs with 8-warp blocks): pulled from one queue
// that runs over the instances in plan order and over each instance's own
// device tile list.  Shared memory is sized for n = kMaxN.
__global__ void __launch_bounds__(32, 8) batch_fused_warp_kernel(PlanPtrs p) {
    __shared__ double sacc[2 * Part<kMaxN>::size * 32];
    __shared__ double krow[2 * 16 * 33];
    __shared__ double kred[64];
    const int lane = threadIdx.x & 31;
    const int nf = p.hdr->nf;
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(&p.hdr->qf, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= nf) break;
        const int j = find_inst(p.pref_ft, p.hdr->ninst, t);
        const InstDesc &d = p.inst[p.order[j]];
        const int slot = t - p.pref_ft[j];  // tile ti, split pc of the instance
        const int npc = d.npc, ti = slot / npc, pc = slot - ti * npc;
        const int PC = (d.nst + npc - 1) / npc, p0 = min(pc * PC, d.nst), p1 = min(p0 + PC, d.nst);
        const size_t PSd = (size_t)(tri(d.n) + 1 + 3 * d.n);
        double *part_b = d.psym, *part_k = d.psym + (size_t)d.nstiles * npc * 2 * PSd * 32;
        double *H = npc > 1 ? d.Hp + (size_t)pc * d.K * d.K : d.H;
        double *S = npc > 1 ? d.Sp + (size_t)pc * d.K * d.K : d.S;
        BATCH_SWITCH(d.n, (fsym_tile<N, true>(slot, d.stiles[ti], d.lc_s, d.K, d.nst, consts_of<N>(d), d.bra,
                                              d.ket, d.C, d.kmap, H, S, part_b, part_k, d.status,
                                              FusedSmem{sacc, krow, kred, nullptr}, false, nullptr, p0, p1)));
    }
}

// Fused pass of every instance: 8-warp blocks, one per SM, persistent over one
// queue of tile groups that runs over the instances in plan order (largest
// tiles first) and over each instance's groups (one 32-row block, 8 consecutive
// ket chunks, one per warp).  The warps of a block work on the same instance and
// bras; the group's bras are staged in shared memory once, each warp's ket
// records too, in two buffers (fsym_tile with BSYNC, SBRA, SKET), and the warps
// meet only at the group's barriers (no barrier per term, as the single-
// instance variant 248).  Shared memory is sized for n = kMaxN.
template <int N> __host__ __device__ constexpr int bfused_warp_smem() {
    return 2 * Part<N>::size * 32 + 2 * 16 * 33 + 64 + 2 * KetLayout<N>::size;
}
constexpr int kBatchFusedSmem = (8 * bfused_warp_smem<kMaxN>() + BraLayout<kMaxN>::size * 32) * 8;

template <int N>
__device__ __forceinline__ void batch_fused_group(const InstDesc &d, int2 gr, double *smem) {
    constexpr int PS = Part<N>::size;
    constexpr int PER_WARP = bfused_warp_smem<N>();
    constexpr int BS = BraLayout<N>::size;
    const int w = threadIdx.x >> 5;
    double *base = smem + w * PER_WARP;
    double *sbra = smem + 8 * PER_WARP;
    const FusedSmem sm{base, base + 2 * PS * 32, base + 2 * PS * 32 + 2 * 16 * 33,
                       base + 2 * PS * 32 + 2 * 16 * 33 + 64};
    const int K = d.K, kb = gr.x, lc = gr.y + w;
    const int last = min(kb * 32 + 31, K - 1);
    const bool idle = lc * d.lc_s > last;
    for (int i = threadIdx.x; i < BS * 32; i += 256) {
        const int f = i >> 5, kk = min(kb * 32 + (i & 31), K - 1);
        sbra[i] = d.bra[(size_t)f * K + kk];
    }
    __syncthreads();
    double *part_b = d.psym, *part_k = d.psym + (size_t)d.nstiles * 2 * PS * 32;
    fsym_tile<N, true, true, true, true, 3>(d.stile_start[kb] + lc, make_int2(kb, lc), d.lc_s, K, d.nst,
                                            consts_of<N>(d), d.bra, d.ket, d.C, d.kmap, d.H, d.S, part_b, part_k,
                                            d.status, sm, idle, sbra);
    __syncthreads();  // sbra and the warps' areas are reused by the next group
}

__global__ void __launch_bounds__(256, 1) batch_fused_kernel(PlanPtrs p) {
    extern __shared__ __align__(16) double smem[];
    __shared__ int gsh;
    const int nf = p.hdr->nf, ninst = p.hdr->ninst;
    for (;;) {
        if (threadIdx.x == 0) gsh = atomicAdd(&p.hdr->qf, 1);
        __syncthreads();
        const int t = gsh;
        __syncthreads();
        if (t >= nf) break;
        const int j = find_inst(p.pref_ft, ninst, t);
        const InstDesc &d = p.inst[p.order[j]];
        const int2 gr = d.bgroups[t - p.pref_ft[j]];
        BATCH_SWITCH(d.n, batch_fused_group<N>(d, gr, smem));
    }
}

// H, S of every instance whose symmetry terms were split: the sum over its
// splits, in a fixed order (before rows / finalize read them).
__global__ void __launch_bounds__(256) batch_hs_reduce_kernel(PlanPtrs p) {
    const int ninst = p.hdr->ninst;
    for (int q = 0; q < ninst; ++q) {
        const InstDesc &d = p.inst[q];
        if (d.npc <= 1) continue;
        const size_t KK = (size_t)d.K * d.K;
        for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < KK; i += (size_t)gridDim.x * blockDim.x) {
            double h = d.Hp[i], s = d.Sp[i];
            for (int pc = 1; pc < d.npc; ++pc) {
                h += d.Hp[pc * KK + i];
                s += d.Sp[pc * KK + i];
            }
            d.H[i] = h;
            d.S[i] = s;
        }
    }
}

// g_H - E g_S of every instance into its part (field-major, chunk 0).
__global__ void __launch_bounds__(256) batch_fsum_kernel(PlanPtrs p) {
    const int ninst = p.hdr->ninst;
    const int total = p.pref_sum[ninst];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int q = find_inst(p.pref_sum, ninst, i);
        const InstDesc &d = p.inst[q];
        const int id = i - p.pref_sum[q];
        const int f = id / d.K, m = id - f * d.K;
        const size_t PSd = (size_t)(tri(d.n) + 1 + 3 * d.n);
        const int npc = d.npc > 1 ? d.npc : 1;
        const double *part_b = d.psym, *part_k = d.psym + (size_t)d.nstiles * npc * 2 * PSd * 32;
        double v = 0.0;
        BATCH_SWITCH(d.n, v = fsym_sum_one<N>(d.stile_start, d.lc_s, d.K, f, m, part_b, part_k, d.scal[0], 0,
                                              0x7fffffff, npc));
        d.part[(size_t)f * d.K + m] = v;
    }
}

// Every instance's status word pair into one array, so one copy reads them all.
__global__ void batch_status_kernel(PlanPtrs p) {
    const int ninst = p.hdr->ninst;
    for (int q = threadIdx.x; q < ninst; q += blockDim.x) {
        p.status_all[2 * q] = p.inst[q].status[0];
        p.status_all[2 * q + 1] = p.inst[q].status[1];
    }
}

__global__ void __launch_bounds__(256) batch_rows_kernel(PlanPtrs p) {
    const int ninst = p.hdr->ninst;
    const int nrows = p.pref_bra[ninst];
    const int lane = threadIdx.x & 31;
    const int wstride = (gridDim.x * blockDim.x) >> 5;
    for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < nrows; r += wstride) {
        const int q = find_inst(p.pref_bra, ninst, r);
        const InstDesc &d = p.inst[q];
        const int i = r - p.pref_bra[q], K = d.K;
        const double *h = d.H + (size_t)i * K, *s = d.S + (size_t)i * K;
        double ah = 0.0, as = 0.0;
        for (int j = lane; j < K; j += 32) {
            ah += h[j] * d.C[j];
            as += s[j] * d.C[j];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ah += __shfl_xor_sync(0xffffffffu, ah, o);
            as += __shfl_xor_sync(0xffffffffu, as, o);
        }
        if (lane == 0) {
            d.rows[i] = ah;
            d.rows[K + i] = as;
        }
    }
}

// E, norm, GRADC per instance (python/outprod.py:65-68, python/make_grad.py:85)
__global__ void __launch_bounds__(256) batch_finalize_kernel(PlanPtrs p) {
    __shared__ double sh[2][8];
    __shared__ double en[2];
    const int ninst = p.hdr->ninst;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int q = blockIdx.x; q < ninst; q += gridDim.x) {
        const InstDesc &d = p.inst[q];
        const int K = d.K;
        double ah = 0.0, as = 0.0;
        for (int i = threadIdx.x; i < K; i += blockDim.x) {
            ah += d.C[i] * d.rows[i];
            as += d.C[i] * d.rows[K + i];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ah += __shfl_xor_sync(0xffffffffu, ah, o);
            as += __shfl_xor_sync(0xffffffffu, as, o);
        }
        if (lane == 0) {
            sh[0][w] = ah;
            sh[1][w] = as;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double th = 0.0, ts = 0.0;
            for (int j = 0; j < (int)(blockDim.x >> 5); ++j) {
                th += sh[0][j];
                ts += sh[1][j];
            }
            const double E = th / ts, nrm = 1.0 / ts;
            d.scal[0] = E;
            d.scal[1] = nrm;
            d.scal[2] = th;
            d.scal[3] = ts;
            if (d.f) d.f[0] = E;
            if (!isfinite(E)) atomicOr(d.status, 2);
            en[0] = E;
            en[1] = nrm;
        }
        __syncthreads();
        const size_t siv = (size_t)K * (d.n * (d.n + 1) / 2 + 3 * d.n);
        for (int i = threadIdx.x; i < K; i += blockDim.x)
            d.g[siv + i] = 2.0 * en[1] * (d.rows[i] - en[0] * d.rows[K + i]);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(32) batch_grad_kernel(PlanPtrs p) {
    const int lane = threadIdx.x & 31;
    const int ng = p.hdr->ng;
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(&p.hdr->qg, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= ng) break;
        const int4 e = p.gtiles[t];
        const InstDesc &d = p.inst[e.x];
        const int nkb = (d.K + 31) / 32;
        int k, lc, l0, l1;
        const int w = e.z * nkb + e.y;  // (kb, lc) as the single-instance kernel numbers it
        if (grad_lane_range(w, lane, nkb, d.lc_g, d.K, k, lc, l0, l1)) {
            bool ok = true;
            BATCH_SWITCH(d.n, ok = (grad_lane<N, double>(BraRef{d.bra + k, (size_t)d.K}, DevKetB{d.ket}, l0, l1,
                                                         d.nst, consts_of<N>(d), 1.0, d.scal[0],
                                                         d.part + (size_t)lc * Part<N>::size * d.K + k,
                                                         (size_t)d.K)));
            if (!ok) flag_inst(d.status, 1, k * d.K + l0);
        }
    }
}

__global__ void __launch_bounds__(256) batch_sum_kernel(PlanPtrs p) {
    const int ninst = p.hdr->ninst;
    const int total = p.pref_sum[ninst];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int q = find_inst(p.pref_sum, ninst, i);
        const InstDesc &d = p.inst[q];
        const size_t id = (size_t)(i - p.pref_sum[q]);
        const size_t stride = (size_t)(p.pref_sum[q + 1] - p.pref_sum[q]);  // PS * K
        double s = d.part[id];
        for (int lc = 1; lc < d.nlc; ++lc) s += d.part[id + lc * stride];
        d.part[id] = s;
    }
}

__global__ void __launch_bounds__(128) batch_reduce_kernel(PlanPtrs p) {
    const int ninst = p.hdr->ninst;
    const int total = p.pref_bra[ninst];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int q = find_inst(p.pref_bra, ninst, i);
        const InstDesc &d = p.inst[q];
        const int k = i - p.pref_bra[q];
        const double sc = d.scal[1] * d.C[k];
        bool fin = true;
        BATCH_SWITCH(d.n, fin = grad_reduce_one<N>(d.part, 1, d.K, d.bra, sc, d.g, k));
        if (!fin) atomicOr(d.status, 2);
    }
}

template <int N> void fill_consts(InstDesc &d, const necg_handle *h) {
    static_assert(sizeof(Consts<N>) <= sizeof(d.cs), "constants do not fit");
    Consts<N> c;
    for (int i = 0; i < N * N; ++i) c.M[i] = h->mass[i];
    c.derive();
    for (int q = 1; q <= N; ++q)
        for (int pp = 0; pp < q; ++pp)
            c.cv[vidx(pp, q)] = 2.0 * h->ncv[pp] * h->ncv[q] / NECG_SQRT_PI;
    for (int i = 0; i < N; ++i) c.q[i] = h->ncv[i + 1];
    c.efs = h->efs;
    c.sqrt8n = sqrt(pow(8.0, N));
    memcpy(d.cs, &c, sizeof(c));
}

}  // namespace necg

using namespace necg;

struct necg_batch {
    int cap_inst = 0, cap_tiles = 0;
    int device = 0, sms = 148;
    int occ_energy = 8, occ_grad = 8, occ_fwarp = 8;  // resident one-warp blocks per SM (persistent kernels)
    int mode = 0;  // of the current plan: 0 ordered, 1 fused lockstep, 2 fused one-warp
    bool fused = false;  // mode of the current plan
    char *d_plan = nullptr;  // device plan buffer
    char *h_plan = nullptr;  // pinned host staging
    size_t plan_bytes = 0;
    PlanPtrs ptrs{};
    std::vector<necg_handle *> active;
    cudaGraph_t graph[3] = {};  // per mode
    cudaGraphExec_t exec[3] = {};
    cudaEvent_t uploaded = nullptr;  // recorded after the last plan upload from h_plan
    int ninst = 0, ne = 0, ng = 0;
};

namespace {
int cfail(cudaError_t e) {
    return e == cudaSuccess ? NECG_OK : (e == cudaErrorMemoryAllocation ? NECG_ERR_ALLOC : NECG_ERR_CUDA);
}
#define BCK(x)                                      \
    do {                                            \
        cudaError_t _e = (x);                       \
        if (_e != cudaSuccess) return cfail(_e);    \
    } while (0)

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

void layout(necg_batch *b, char *base, PlanPtrs &p, size_t *total) {
    size_t off = 0;
    p.hdr = (PlanHdr *)(base + off);
    off = align_up(off + sizeof(PlanHdr), 256);
    p.inst = (InstDesc *)(base + off);
    off = align_up(off + sizeof(InstDesc) * b->cap_inst, 256);
    p.pref_bra = (int *)(base + off);
    off = align_up(off + sizeof(int) * (b->cap_inst + 1), 256);
    p.pref_ket = (int *)(base + off);
    off = align_up(off + sizeof(int) * (b->cap_inst + 1), 256);
    p.pref_sum = (int *)(base + off);
    off = align_up(off + sizeof(int) * (b->cap_inst + 1), 256);
    p.pref_ft = (int *)(base + off);
    off = align_up(off + sizeof(int) * (b->cap_inst + 1), 256);
    p.order = (int *)(base + off);
    off = align_up(off + sizeof(int) * (b->cap_inst + 1), 256);
    p.etiles = (int4 *)(base + off);
    off = align_up(off + sizeof(int4) * b->cap_tiles, 256);
    p.gtiles = (int4 *)(base + off);
    off = align_up(off + sizeof(int4) * b->cap_tiles, 256);
    p.status_all = (int *)(base + off);
    off = align_up(off + sizeof(int) * 2 * b->cap_inst, 256);
    if (total) *total = off;
}

// mode: 0 ordered, 1 fused (lockstep blocks), 2 fused (one-warp blocks)
void launch_step(necg_batch *b, cudaStream_t st, int mode) {
    const PlanPtrs &p = b->ptrs;
    const int g = b->sms;
    batch_reset_kernel<<<1, 256, 0, st>>>(p);
    batch_prep_kernel<<<g * 4, 128, 0, st>>>(p);
    if (mode) {
        if (mode == 2) {
            batch_fused_warp_kernel<<<g * b->occ_fwarp, 32, 0, st>>>(p);
            batch_hs_reduce_kernel<<<g * 2, 256, 0, st>>>(p);
        } else {
            batch_fused_kernel<<<g, 256, kBatchFusedSmem, st>>>(p);
        }
        batch_rows_kernel<<<g * 4, 256, 0, st>>>(p);
        batch_finalize_kernel<<<g, 256, 0, st>>>(p);
        batch_fsum_kernel<<<g * 4, 256, 0, st>>>(p);
    } else {
        batch_energy_kernel<<<g * b->occ_energy, 32, 0, st>>>(p);
        batch_rows_kernel<<<g * 4, 256, 0, st>>>(p);
        batch_finalize_kernel<<<g, 256, 0, st>>>(p);
        batch_grad_kernel<<<g * b->occ_grad, 32, 0, st>>>(p);
        batch_sum_kernel<<<g * 4, 256, 0, st>>>(p);
    }
    batch_reduce_kernel<<<g * 2, 128, 0, st>>>(p);
    batch_status_kernel<<<1, 256, 0, st>>>(p);
}

int capture(necg_batch *b, int mode) {
    if (b->exec[mode]) cudaGraphExecDestroy(b->exec[mode]);
    if (b->graph[mode]) cudaGraphDestroy(b->graph[mode]);
    b->exec[mode] = nullptr;
    b->graph[mode] = nullptr;
    cudaStream_t cap;
    BCK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        launch_step(b, cap, mode);
        e = cudaStreamEndCapture(cap, &b->graph[mode]);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec[mode], b->graph[mode], 0);
    cudaStreamDestroy(cap);
    return cfail(e);
}
}  // namespace

extern "C" {

int necg_batch_create(int max_instances, int max_tiles, necg_batch **out) {
    if (!out || max_instances < 1 || max_tiles < 1) return NECG_ERR_ARG;
    *out = nullptr;
    necg_batch *b = new necg_batch();
    b->cap_inst = max_instances;
    b->cap_tiles = max_tiles;
    cudaGetDevice(&b->device);
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
    // persistent grids: exactly the resident capacity
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->occ_energy, batch_energy_kernel, 32, 0) != cudaSuccess ||
        b->occ_energy < 1)
        b->occ_energy = 8;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->occ_grad, batch_grad_kernel, 32, 0) != cudaSuccess ||
        b->occ_grad < 1)
        b->occ_grad = 8;
    PlanPtrs tmp{};
    layout(b, nullptr, tmp, &b->plan_bytes);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->occ_fwarp, batch_fused_warp_kernel, 32, 0) != cudaSuccess ||
        b->occ_fwarp < 1)
        b->occ_fwarp = 8;
    // the lockstep fused kernel's shared memory (one 8-warp block per SM) needs the opt-in
    cudaError_t e = cudaFuncSetAttribute(batch_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kBatchFusedSmem);
    if (e == cudaSuccess) e = cudaMalloc((void **)&b->d_plan, b->plan_bytes);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&b->h_plan, b->plan_bytes);
    if (e == cudaSuccess) e = cudaMemset(b->d_plan, 0, b->plan_bytes);
    if (e != cudaSuccess) {
        if (b->d_plan) cudaFree(b->d_plan);
        if (b->h_plan) cudaFreeHost(b->h_plan);
        delete b;
        return cfail(e);
    }
    layout(b, b->d_plan, b->ptrs, nullptr);
    *out = b;
    return NECG_OK;
}

int necg_batch_destroy(necg_batch *b) {
    if (!b) return NECG_ERR_ARG;
    cudaSetDevice(b->device);
    for (int m = 0; m < 3; ++m) {
        if (b->exec[m]) cudaGraphExecDestroy(b->exec[m]);
        if (b->graph[m]) cudaGraphDestroy(b->graph[m]);
    }
    if (b->uploaded) cudaEventDestroy(b->uploaded);
    cudaFree(b->d_plan);
    cudaFreeHost(b->h_plan);
    delete b;
    return NECG_OK;
}

int necg_batch_plan(necg_batch *b, int count, necg_handle *const *hs, const int *Ks,
                    const double *const *x_dev, double *const *g_dev, double *const *f_dev,
                    void *stream) {
    necg::TraceRange trace("necg_batch_plan");
    if (!b || count < 0 || count > b->cap_inst || (count > 0 && (!hs || !Ks || !x_dev || !g_dev)))
        return NECG_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    BCK(cudaSetDevice(b->device));
    // the pinned staging buffer may still be read by this batch's previous upload
    if (b->uploaded) BCK(cudaEventSynchronize(b->uploaded));
    PlanPtrs hp{};
    layout(b, b->h_plan, hp, nullptr);
    struct Cost {
        double c;
        int4 t;
    };
    std::vector<Cost> et, gt;
    std::vector<double> fcost(count > 0 ? count : 1, 0.0);
    static const std::vector<long long> flops_fused = [] {
        std::vector<long long> v(kMaxN + 1, 0);
        for (int n = 1; n <= kMaxN; ++n) v[n] = necg_term_flops(n, 3, nullptr);
        return v;
    }();
    hp.pref_bra[0] = hp.pref_ket[0] = hp.pref_sum[0] = 0;
    bool fused = count > 0;
    for (int q = 0; q < count; ++q) {
        if (!hs[q] || !hs[q]->sym_ok || hs[q]->n > kMaxN) fused = false;
    }
    for (int q = 0; q < count; ++q) {
        necg_handle *h = hs[q];
        const int K = Ks[q];
        if (!h || K < 1 || K > h->K_max || h->lc_g < 4) return NECG_ERR_ARG;
        if (h->n < 1 || h->n > kMaxN) return NECG_ERR_UNSUPPORTED;
        InstDesc &d = hp.inst[q];
        memset(&d, 0, sizeof(d));
        const int n = h->n;
        const size_t siv = (size_t)K * (n * (n + 1) / 2 + 3 * n);
        d.n = n;
        d.K = K;
        d.nst = h->nst;
        d.lc_e = h->lc_e;
        d.lc_g = h->lc_g;
        d.nlc = (K + h->lc_g - 1) / h->lc_g;
        d.iv = x_dev[q];
        d.C = x_dev[q] + siv;
        d.bra = h->d_bra;
        d.ket = h->d_ket;
        d.part = h->d_part;
        d.H = h->d_H;
        d.S = h->d_S;
        d.rows = h->d_rows;
        d.scal = h->d_scal;
        d.g = g_dev[q];
        d.f = f_dev ? f_dev[q] : nullptr;
        d.sml = h->d_sml;
        d.sms = h->d_sms;
        d.scvv = h->d_scvv;
        d.status = h->d_status;
        BATCH_SWITCH(n, fill_consts<N>(d, h));
        if (fused) {
            int rc = prepare_fused(h, K, st);
            if (rc) return rc;
            d.lc_s = h->lc_s;
            d.nstiles = h->nstiles;
            d.pinv = h->d_pinv;
            d.stile_start = h->d_stile_start;
            d.psym = h->d_psym;
            d.kmap = KetMap{h->d_kcnt, h->d_ksrc, h->d_kcoef, h->kmaxnz};
            d.stiles = h->d_stiles;
            d.bgroups = h->d_bgroups;
            d.nbgroups = h->nbgroups;
            d.npc = 1;  // set below for the one-warp kernel
            d.Hp = h->d_Hp;
            d.Sp = h->d_Sp;
        }
        const int ps = tri(n) + 1 + 3 * n;
        hp.pref_bra[q + 1] = hp.pref_bra[q] + K;
        hp.pref_ket[q + 1] = hp.pref_ket[q] + K * h->nst;
        hp.pref_sum[q + 1] = hp.pref_sum[q] + ps * K;
        const int nkb = (K + 31) / 32;
        if (fused) {  // tiles come from the instance's device list; only its cost is needed here
            fcost[q] = (double)flops_fused[n] * h->nst * d.lc_s;
            continue;
        }
        const long long fe = necg_term_flops(n, 0, nullptr), fg = necg_term_flops(n, 1, nullptr);
        for (int kb = 0; kb < nkb; ++kb)
            for (int lc = 0; lc * d.lc_e <= kb * 32 + 31 && lc * d.lc_e < K; ++lc)
                et.push_back({(double)fe * h->nst * d.lc_e, make_int4(q, kb, lc, 0)});
        for (int lc = 0; lc < d.nlc; ++lc)
            for (int kb = 0; kb < nkb; ++kb)
                gt.push_back({(double)fg * h->nst * d.lc_g, make_int4(q, kb, lc, 0)});
    }
    long long nf = 0;
    bool fine = false;
    if (fused) {  // fused queue: instances by decreasing tile cost, each over its own groups / tiles
        for (int q = 0; q < count; ++q) hp.order[q] = q;
        std::stable_sort(hp.order, hp.order + count, [&](int a, int c) { return fcost[a] > fcost[c]; });
        long long ng = 0;
        for (int q = 0; q < count; ++q) ng += hp.inst[q].nbgroups;
        fine = ng < 4LL * b->sms;  // too few groups to fill the SMs with 8-warp blocks
        // the one-warp kernel splits each instance's symmetry terms as its handle does
        // (its partial buffers and H, S split buffers are sized for that)
        if (fine)
            for (int q = 0; q < count; ++q) hp.inst[q].npc = fused_splits(hs[q]);
        hp.pref_ft[0] = 0;
        for (int j = 0; j < count; ++j) {
            const InstDesc &dj = hp.inst[hp.order[j]];
            nf += fine ? (long long)dj.nstiles * dj.npc : dj.nbgroups;
            if (nf > 0x7fffffff) return NECG_ERR_CAPACITY;
            hp.pref_ft[j + 1] = (int)nf;
        }
    }
    if ((int)et.size() > b->cap_tiles || (int)gt.size() > b->cap_tiles) return NECG_ERR_CAPACITY;
    auto by_cost = [](const Cost &a, const Cost &c) { return a.c > c.c; };
    std::stable_sort(et.begin(), et.end(), by_cost);
    std::stable_sort(gt.begin(), gt.end(), by_cost);
    for (size_t i = 0; i < et.size(); ++i) hp.etiles[i] = et[i].t;
    for (size_t i = 0; i < gt.size(); ++i) hp.gtiles[i] = gt[i].t;
    hp.hdr->ninst = count;
    hp.hdr->ne = fused ? 0 : (int)et.size();
    hp.hdr->ng = (int)gt.size();
    hp.hdr->nf = fused ? (int)nf : 0;
    hp.hdr->fine = fine ? 1 : 0;
    hp.hdr->qe = hp.hdr->qg = hp.hdr->qf = 0;
    b->fused = fused;
    b->mode = fused ? (fine ? 2 : 1) : 0;
    b->ninst = count;
    b->ne = (int)et.size();
    b->ng = (int)gt.size();
    b->active.assign(hs, hs + count);
    // upload only what this plan uses: header, instance table and prefixes,
    // then the used part of each tile queue
    const size_t head = (size_t)((char *)hp.etiles - b->h_plan);
    const size_t off_g = (size_t)((char *)hp.gtiles - b->h_plan);
    BCK(cudaMemcpyAsync(b->d_plan, b->h_plan, head + et.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
    if (!gt.empty())
        BCK(cudaMemcpyAsync(b->d_plan + off_g, b->h_plan + off_g, gt.size() * sizeof(int4),
                            cudaMemcpyHostToDevice, st));
    if (!b->uploaded) BCK(cudaEventCreateWithFlags(&b->uploaded, cudaEventDisableTiming));
    BCK(cudaEventRecord(b->uploaded, st));
    return NECG_OK;
}

int necg_batch_step(necg_batch *b, void *stream) {
    necg::TraceRange trace("necg_batch_step");
    if (!b) return NECG_ERR_ARG;
    BCK(cudaSetDevice(b->device));
    launch_step(b, (cudaStream_t)stream, b->mode);
    return cfail(cudaGetLastError());
}

int necg_batch_graph(necg_batch *b, void *stream) {
    if (!b) return NECG_ERR_ARG;
    BCK(cudaSetDevice(b->device));
    (void)stream;
    return capture(b, b->mode);
}

int necg_batch_replay(necg_batch *b, void *stream) {
    necg::TraceRange trace("necg_batch_replay");
    if (!b) return NECG_ERR_ARG;
    BCK(cudaSetDevice(b->device));
    const int mode = b->mode;
    if (!b->exec[mode]) {  // the graph of this plan's mode was not captured yet
        int rc = capture(b, mode);
        if (rc) return rc;
    }
    BCK(cudaGraphLaunch(b->exec[mode], (cudaStream_t)stream));
    return NECG_OK;
}

int necg_batch_status_async(necg_batch *b, int *flags_host, void *stream) {
    if (!b || (b->ninst > 0 && !flags_host)) return NECG_ERR_ARG;
    BCK(cudaSetDevice(b->device));
    if (b->ninst > 0)
        BCK(cudaMemcpyAsync(flags_host, b->ptrs.status_all, sizeof(int) * 2 * b->ninst, cudaMemcpyDeviceToHost,
                            (cudaStream_t)stream));
    return NECG_OK;
}

int necg_batch_status(necg_batch *b, int *status_out, void *stream) {
    if (!b || (b->ninst > 0 && !status_out)) return NECG_ERR_ARG;
    BCK(cudaSetDevice(b->device));
    cudaStream_t st = (cudaStream_t)stream;
    std::vector<int> tmp(2 * b->ninst);
    for (int q = 0; q < b->ninst; ++q)
        BCK(cudaMemcpyAsync(&tmp[2 * q], b->active[q]->d_status, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    BCK(cudaStreamSynchronize(st));
    int worst = NECG_OK;
    for (int q = 0; q < b->ninst; ++q) {
        const int fl = tmp[2 * q];
        const int code = (fl & 1) ? NECG_ERR_NOT_PD : (fl & 2) ? NECG_ERR_NONFINITE : NECG_OK;
        status_out[q] = code;
        if (code && !worst) worst = code;
    }
    return worst;
}

}  // extern "C"
