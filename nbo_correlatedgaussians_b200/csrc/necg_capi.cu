// necg_capi.cu -- the extern "C" boundary declared in include/necg.h.
//
// A handle owns one particle system's constants (mass, charges, symmetry set)
// on the device plus the workspace one evaluation needs for bases of up to
// K_max functions:
//   bra   BraLayout<n>::size * K_max       per-basis data (structure of arrays)
//   ket   KetLayout<n>::size * K_max * nst per-(l, P) ket records
//   part  part_stride(n) * K_max * ceil(K_max / lc_grad)   gradient tile partials
//   H, S  K_max^2 each (used when the caller passes no H/S)
//   rows  2 K_max, scal 4, x/g staging for the host-pointer entry point
// Nothing is allocated after necg_create, so every device-pointer entry point
// is stream-ordered and capturable in a CUDA graph once tiles for K exist.
//
// Handle memory comes from one stream-ordered pool per device (cudaMemPool_t,
// blocks kept for reuse), allocated and freed on the library's own
// non-blocking stream of that device, or on the caller's stream when an
// evaluation grows a buffer.  Unlike cudaMalloc / cudaFree, creating and
// destroying a handle then never waits for work that other streams have in
// flight, so a server can admit and retire runs while its steps keep running.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>
#include <vector>

#include "necg_handle.h"
#include "necg_kernels.cuh"
#include "necg_math.cuh"
#include "necg_trace.h"

using necg::LaunchArgs;

namespace {

// Status code of the two device status words (flags, first failing pair).
int status_code(const int st[2], long long *bad_pair) {
    if (bad_pair) *bad_pair = st[1] == 0x7fffffff ? -1 : (long long)st[1];
    if (st[0] & 1) return NECG_ERR_NOT_PD;
    if (st[0] & 2) return NECG_ERR_NONFINITE;
    if (st[0] & 4) return NECG_ERR_ARG;
    return NECG_OK;
}

int cuda_fail(cudaError_t e) {
    if (e == cudaSuccess) return NECG_OK;
    return e == cudaErrorMemoryAllocation ? NECG_ERR_ALLOC : NECG_ERR_CUDA;
}

#define CK(x)                                  \
    do {                                       \
        cudaError_t _e = (x);                  \
        if (_e != cudaSuccess) return cuda_fail(_e); \
    } while (0)

// The per-device pool and stream, made on first use with that device current.
struct DevicePool {
    std::once_flag once;
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
    cudaError_t err = cudaSuccess;
};
DevicePool g_pools[64];

cudaError_t device_pool(int dev, cudaMemPool_t *pool, cudaStream_t *stream) {
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    DevicePool &d = g_pools[dev];
    std::call_once(d.once, [&] {
        cudaMemPoolProps props;
        memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        d.err = cudaMemPoolCreate(&d.pool, &props);
        if (d.err == cudaSuccess) {
            uint64_t keep = UINT64_MAX;  // freed blocks stay in the pool for the next handle
            d.err = cudaMemPoolSetAttribute(d.pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        if (d.err == cudaSuccess) d.err = cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking);
    });
    *pool = d.pool;
    *stream = d.stream;
    return d.err;
}

// Stream-ordered allocation from the handle's device pool on stream st (the
// library stream when st is null).
template <typename T> cudaError_t pool_alloc(necg_handle *h, T **p, size_t bytes, cudaStream_t st = nullptr) {
    cudaMemPool_t pool;
    cudaStream_t ls;
    cudaError_t e = device_pool(h->device, &pool, &ls);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync((void **)p, bytes, pool, st ? st : ls);
    if (e != cudaSuccess) *p = nullptr;
    return e;
}

void pool_free(necg_handle *h, void *p, cudaStream_t st = nullptr) {
    if (!p) return;
    cudaMemPool_t pool;
    cudaStream_t ls;
    if (device_pool(h->device, &pool, &ls) == cudaSuccess) cudaFreeAsync(p, st ? st : ls);
}

cudaStream_t lib_stream(necg_handle *h) {
    cudaMemPool_t pool;
    cudaStream_t ls = nullptr;
    device_pool(h->device, &pool, &ls);
    return ls;
}

template <typename T> int dalloc(necg_handle *h, T **p, size_t count) {
    size_t bytes = count * sizeof(T);
    if (bytes == 0) bytes = 16;
    cudaError_t e = pool_alloc(h, p, bytes);
    if (e != cudaSuccess) return cuda_fail(e);
    h->ws_bytes += (long long)bytes;
    return NECG_OK;
}

// Phase event i of the evaluation (profiling).  While the stream is being
// captured it is recorded as an external event, so that the captured graph
// records it when it runs.
void mark(necg_handle *h, int i, cudaStream_t st) {
    if (!h->profile) return;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cap);
    if (cap == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(h->ev[i], st, cudaEventRecordExternal);
    else cudaEventRecord(h->ev[i], st);
}

void free_all(necg_handle *h) {
    for (cudaEvent_t &e : h->ev)
        if (e) cudaEventDestroy(e);
    void *ptrs[] = {h->d_sml, h->d_sms, h->d_scvv, h->d_bra, h->d_ket, h->d_part, h->d_H,
                    h->d_S, h->d_rows, h->d_scal, h->d_x, h->d_g, h->d_f, h->d_status,
                    h->d_tiles, h->d_pinv, h->d_kcnt, h->d_ksrc, h->d_kcoef, h->d_stiles,
                    h->d_stile_start, h->d_psym, h->d_sgroups, h->d_qcount, h->d_bgroups,
                    h->d_Hp, h->d_Sp, h->d_xsym, h->d_urange};
    for (void *p : ptrs) pool_free(h, p);
}

// Energy tiles over the lower triangle: (kb, lc) with lc * LC <= kb * 32 + 31.
int ensure_tiles(necg_handle *h, int K, cudaStream_t st) {
    if (h->tiles_K == K && h->tiles_lc == h->lc_e) return NECG_OK;
    std::vector<int2> t;
    const int nkb = (K + 31) / 32;
    for (int kb = 0; kb < nkb; ++kb) {
        const int kmax = kb * 32 + 31;
        for (int lc = 0; lc * h->lc_e <= kmax && lc * h->lc_e < K; ++lc) t.push_back(make_int2(kb, lc));
    }
    if ((int)t.size() > h->tiles_cap) {
        pool_free(h, h->d_tiles, st);
        h->d_tiles = nullptr;
        CK(pool_alloc(h, &h->d_tiles, t.size() * sizeof(int2), st));
        h->tiles_cap = (int)t.size();
    }
    CK(cudaMemcpyAsync(h->d_tiles, t.data(), t.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    h->tiles_K = K;
    ++h->gversion;  // buffers and lists a captured graph may hold changed
    h->tiles_lc = h->lc_e;
    h->ntiles = (int)t.size();
    return NECG_OK;
}

// Lower-triangle tiles of chunk LC for the symmetric pass, plus the first tile
// of each 32-row block; the partial buffer grows here if this K and LC need more.
// mult = 2 for the fused pass (H and S partials kept apart), 1 otherwise; the
// fused pass with npc splits needs npc partial slots per tile and npc K x K
// buffers for H and S.
int ensure_sym_tiles(necg_handle *h, int K, cudaStream_t st, int mult) {
    const int PS = necg::part_stride(h->n);
    const int gw = necg::fused_block_warps(h->minb_s);  // tiles per group of the lockstep-block pass
    const int npc = mult == 2 ? necg::fused_splits(h) : 1;
    const size_t hp_need = npc > 1 ? (size_t)npc * K * K : 0;
    if (hp_need > h->hp_cap) {
        pool_free(h, h->d_Hp, st);
        pool_free(h, h->d_Sp, st);
        h->d_Hp = h->d_Sp = nullptr;
        h->hp_cap = 0;
        CK(pool_alloc(h, &h->d_Hp, hp_need * sizeof(double), st));
        CK(pool_alloc(h, &h->d_Sp, hp_need * sizeof(double), st));
        ++h->gversion;
        h->ws_bytes += (long long)(2 * hp_need * sizeof(double));
        h->hp_cap = hp_need;
    }
    if (h->stiles_K == K && h->stiles_lc == h->lc_s && h->sgroups_w == gw &&
        (size_t)h->nstiles * PS * (32 + h->lc_s) * mult * npc <= h->psym_cap)
        return NECG_OK;
    std::vector<int2> t;
    std::vector<int> start;
    const int nkb = (K + 31) / 32, LC = h->lc_s;
    for (int kb = 0; kb < nkb; ++kb) {
        start.push_back((int)t.size());
        const int last = kb * 32 + 31 < K - 1 ? kb * 32 + 31 : K - 1;
        for (int lc = 0; lc <= last / LC; ++lc) t.push_back(make_int2(kb, lc));
    }
    start.push_back((int)t.size());
    if ((int)t.size() > h->stiles_cap) {
        pool_free(h, h->d_stiles, st);
        h->d_stiles = nullptr;
        CK(pool_alloc(h, &h->d_stiles, t.size() * sizeof(int2), st));
        h->stiles_cap = (int)t.size();
    }
    if (!h->d_stile_start) CK(pool_alloc(h, &h->d_stile_start, ((h->K_max + 31) / 32 + 2) * sizeof(int), st));
    const size_t need = t.size() * (size_t)PS * (32 + LC) * mult * npc;
    if (need > h->psym_cap) {
        pool_free(h, h->d_psym, st);
        h->d_psym = nullptr;
        CK(pool_alloc(h, &h->d_psym, need * sizeof(double), st));
        h->ws_bytes += (long long)((need - h->psym_cap) * sizeof(double));
        h->psym_cap = need;
    }
    std::vector<int2> groups;  // gw consecutive ket chunks of one row block, largest blocks first
    for (int kb = nkb - 1; kb >= 0; --kb) {
        const int ntk = start[kb + 1] - start[kb];
        for (int lc0 = 0; lc0 < ntk; lc0 += gw) groups.push_back(necg::sgroup_pack(kb, lc0, 0, 1));
    }
    // The groups are equal work, one block per SM takes them from the queue, so
    // the last round runs G mod SMs groups while the other SMs idle: split each
    // of those groups into `parts` units over the symmetry terms (as many as
    // keep the round within one unit per SM, at most 8; the kernel gives the
    // parts balanced ranges of terms), so the last round is a part of a group
    // long.
    {
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
        const int G = (int)groups.size();
        const int T = G % sms;
        int parts = T > 0 ? sms / T : 1;
        if (parts > 8) parts = 8;
        if (parts > h->nst) parts = h->nst;
        // the lockstep pass writes bra partials per queue unit into the slots
        // sized for the tiles: G - T + T parts units must not exceed them
        if (T > 0 && parts > 1 + ((int)t.size() - G) / T) parts = 1 + ((int)t.size() - G) / T;
        h->sg_ntail = 0;
        h->sg_parts = 1;
        h->sg_tail0 = G;
        if (parts >= 2) {
            std::vector<int2> tail(groups.end() - T, groups.end());
            groups.resize(G - T);
            for (const int2 &g : tail)
                for (int q = 0; q < parts; ++q)
                    groups.push_back(necg::sgroup_pack(g.x, necg::sgroup_lc0(g), q, parts));
            h->sg_tail0 = G - T;
            h->sg_ntail = T;
            h->sg_parts = parts;
            const size_t xneed = (size_t)T * gw * (parts - 1) * necg::fsym_tail_slot(PS, LC);
            if (xneed > h->xsym_cap) {
                pool_free(h, h->d_xsym, st);
                h->d_xsym = nullptr;
                h->xsym_cap = 0;
                CK(pool_alloc(h, &h->d_xsym, xneed * sizeof(double), st));
                h->ws_bytes += (long long)(xneed * sizeof(double));
                h->xsym_cap = xneed;
            }
        }
    }
    if ((int)groups.size() > h->sgroups_cap) {
        pool_free(h, h->d_sgroups, st);
        h->d_sgroups = nullptr;
        CK(pool_alloc(h, &h->d_sgroups, groups.size() * sizeof(int2), st));
        h->sgroups_cap = (int)groups.size();
    }
    if (!h->d_qcount) CK(pool_alloc(h, &h->d_qcount, sizeof(int), st));
    // each row block's queue units are contiguous (blocks in decreasing order,
    // a split group's parts next to each other)
    std::vector<int2> urange(nkb, make_int2(0, 0));
    for (int u = 0; u < (int)groups.size(); ++u) {
        int2 &r = urange[groups[u].x];
        if (r.y == 0) r.x = u;
        r.y = u + 1;
    }
    if (nkb > h->urange_cap) {
        pool_free(h, h->d_urange, st);
        h->d_urange = nullptr;
        CK(pool_alloc(h, &h->d_urange, nkb * sizeof(int2), st));
        h->urange_cap = nkb;
    }
    CK(cudaMemcpyAsync(h->d_urange, urange.data(), nkb * sizeof(int2), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(h->d_sgroups, groups.data(), groups.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
    h->nsgroups = (int)groups.size();
    h->sgroups_w = gw;
    std::vector<int2> bgroups;  // width 8, for the batched step
    for (int kb = nkb - 1; kb >= 0; --kb) {
        const int ntk = start[kb + 1] - start[kb];
        for (int lc0 = 0; lc0 < ntk; lc0 += 8) bgroups.push_back(make_int2(kb, lc0));
    }
    if ((int)bgroups.size() > h->bgroups_cap) {
        pool_free(h, h->d_bgroups, st);
        h->d_bgroups = nullptr;
        CK(pool_alloc(h, &h->d_bgroups, bgroups.size() * sizeof(int2), st));
        h->bgroups_cap = (int)bgroups.size();
    }
    CK(cudaMemcpyAsync(h->d_bgroups, bgroups.data(), bgroups.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
    h->nbgroups = (int)bgroups.size();
    CK(cudaMemcpyAsync(h->d_stiles, t.data(), t.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(h->d_stile_start, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    h->stiles_K = K;
    ++h->gversion;
    h->stiles_lc = LC;
    h->nstiles = (int)t.size();
    return NECG_OK;
}

}  // namespace

int necg::prepare_fused(necg_handle *h, int K, cudaStream_t st) {
    if (!h || !h->sym_ok) return NECG_ERR_UNSUPPORTED;
    CK(cudaSetDevice(h->device));
    return ensure_sym_tiles(h, K, st, 2);
}

namespace {

// Inverse of each symmetry term (sml and sms both inverted) and the map of a
// ket gradient from P's frame to the basis function's frame.  Sets sym_ok
// when every term's inverse is in the set and n <= 5.
int setup_symmetric(necg_handle *h) {
    const int n = h->n, nst = h->nst, m = 3 * n;
    if (n > 5) return NECG_OK;
    std::vector<int> pinv(nst, -1);
    for (int p = 0; p < nst; ++p)
        for (int q = 0; q < nst && pinv[p] < 0; ++q) {
            bool ok = true;
            for (int i = 0; i < n && ok; ++i)
                for (int j = 0; j < n && ok; ++j) {
                    double s = 0.0;
                    for (int k = 0; k < n; ++k) s += h->sml[(size_t)p * n * n + i * n + k] * h->sml[(size_t)q * n * n + k * n + j];
                    ok = fabs(s - (i == j ? 1.0 : 0.0)) < 1e-12;
                }
            for (int i = 0; i < m && ok; ++i)
                for (int j = 0; j < m && ok; ++j) {
                    double s = 0.0;
                    for (int k = 0; k < m; ++k) s += h->sms[(size_t)p * m * m + i * m + k] * h->sms[(size_t)q * m * m + k * m + j];
                    ok = fabs(s - (i == j ? 1.0 : 0.0)) < 1e-12;
                }
            if (ok) pinv[p] = q;
        }
    for (int p = 0; p < nst; ++p)
        if (pinv[p] < 0) return NECG_OK;  // not closed under inverse: ordered pass only
    const int T = n * (n + 1) / 2, PS = T + 1 + m;
    std::vector<std::vector<std::pair<int, double>>> rows((size_t)nst * PS);
    for (int p = 0; p < nst; ++p) {
        const double *P = &h->sml[(size_t)p * n * n];
        const double *Sm = &h->sms[(size_t)p * m * m];
        for (int a = 0; a < n; ++a)
            for (int b = 0; b <= a; ++b) {  // (sml G' sml^T)_ab
                std::vector<double> coef(T, 0.0);
                for (int cc = 0; cc < n; ++cc)
                    for (int d = 0; d < n; ++d) coef[necg::sx(cc, d)] += P[a * n + cc] * P[b * n + d];
                auto &row = rows[(size_t)p * PS + necg::sx(a, b)];
                for (int s = 0; s < T; ++s)
                    if (coef[s] != 0.0) row.push_back({s, coef[s]});
            }
        rows[(size_t)p * PS + T].push_back({T, 1.0});
        for (int r = 0; r < m; ++r) {  // (sms^T g')_r
            auto &row = rows[(size_t)p * PS + T + 1 + r];
            for (int cc = 0; cc < m; ++cc)
                if (Sm[cc * m + r] != 0.0) row.push_back({T + 1 + cc, Sm[cc * m + r]});
        }
    }
    int maxnz = 1;
    for (auto &r : rows) maxnz = (int)r.size() > maxnz ? (int)r.size() : maxnz;
    std::vector<int> cnt(rows.size()), src(rows.size() * maxnz, 0);
    std::vector<double> coef(rows.size() * maxnz, 0.0);
    for (size_t e = 0; e < rows.size(); ++e) {
        cnt[e] = (int)rows[e].size();
        for (size_t i = 0; i < rows[e].size(); ++i) {
            src[e * maxnz + i] = rows[e][i].first;
            coef[e * maxnz + i] = rows[e][i].second;
        }
    }
    int rc = NECG_OK;
    if (!rc) rc = dalloc(h, &h->d_pinv, (size_t)nst);
    if (!rc) rc = dalloc(h, &h->d_kcnt, cnt.size());
    if (!rc) rc = dalloc(h, &h->d_ksrc, src.size());
    if (!rc) rc = dalloc(h, &h->d_kcoef, coef.size());
    if (rc) return rc;
    cudaStream_t ls = lib_stream(h);
    CK(cudaMemcpyAsync(h->d_pinv, pinv.data(), nst * sizeof(int), cudaMemcpyHostToDevice, ls));
    CK(cudaMemcpyAsync(h->d_kcnt, cnt.data(), cnt.size() * sizeof(int), cudaMemcpyHostToDevice, ls));
    CK(cudaMemcpyAsync(h->d_ksrc, src.data(), src.size() * sizeof(int), cudaMemcpyHostToDevice, ls));
    CK(cudaMemcpyAsync(h->d_kcoef, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice, ls));
    CK(cudaStreamSynchronize(ls));  // the host vectors above end with this scope
    h->kmaxnz = maxnz;
    h->sym_ok = true;
    h->grad_mode = 1;
    return NECG_OK;
}

LaunchArgs base_args(necg_handle *h, int K) {
    LaunchArgs a;
    memset(&a, 0, sizeof(a));
    a.n = h->n;
    a.K = K;
    a.nst = h->nst;
    a.efs = h->efs;
    a.mass_h = h->mass.data();
    a.ncv_h = h->ncv.data();
    a.sml = h->d_sml;
    a.sms = h->d_sms;
    a.scvv = h->d_scvv;
    a.bra = h->d_bra;
    a.ket = h->d_ket;
    a.tiles = h->d_tiles;
    a.ntiles = h->ntiles;
    a.LC_e = h->lc_e;
    a.LC_g = h->lc_g;
    a.minb_e = h->minb_e;
    a.minb_g = h->minb_g;
    a.rows = h->d_rows;
    a.scal = h->d_scal;
    a.part = h->d_part;
    a.status = h->d_status;
    a.lam = 1.0;
    a.pinv = h->d_pinv;
    a.kmap = necg::KetMap{h->d_kcnt, h->d_ksrc, h->d_kcoef, h->kmaxnz};
    a.stiles = h->d_stiles;
    a.stile_start = h->d_stile_start;
    a.nstiles = h->nstiles;
    a.LC_s = h->lc_s;
    a.minb_s = h->minb_s;
    a.psym = h->d_psym;
    a.sgroups = h->d_sgroups;
    a.nsgroups = h->nsgroups;
    a.qcount = h->d_qcount;
    a.xsym = h->d_xsym;
    a.sg_tail0 = h->sg_tail0;
    a.sg_ntail = h->sg_ntail;
    a.sg_parts = h->sg_parts;
    a.urange = h->d_urange;
    return a;
}

// The gradient passes after E and norm are in scal: symmetric (unordered pairs)
// when available, ordered otherwise.  (Mode 2 fuses the symmetric pass with the
// energy pass of necg_outprod; here H and S are already known, so the
// symmetric pass alone is used.)
int launch_gradient(necg_handle *h, LaunchArgs &a, cudaStream_t st) {
    if (h->grad_mode >= 1) {
        int rc = ensure_sym_tiles(h, a.K, st, h->grad_mode == 2 ? 2 : 1);
        if (rc) return rc;
        a.stiles = h->d_stiles;
        a.stile_start = h->d_stile_start;
        a.nstiles = h->nstiles;
        a.LC_s = h->lc_s;
        a.psym = h->d_psym;
        mark(h, 3, st);
        necg::launch_gsym(a, st);
        mark(h, 4, st);
        necg::launch_gsym_reduce(a, st);
        mark(h, 5, st);
        return NECG_OK;
    }
    mark(h, 3, st);
    necg::launch_grad_tiles(a, st);
    mark(h, 4, st);
    necg::launch_grad_reduce(a, st);
    mark(h, 5, st);
    return NECG_OK;
}

int check_K(necg_handle *h, int K) {
    if (!h) return NECG_ERR_ARG;
    if (K < 1) return NECG_ERR_ARG;
    if (K > h->K_max) return NECG_ERR_CAPACITY;
    return NECG_OK;
}

int begin(necg_handle *h, cudaStream_t st) {
    CK(cudaSetDevice(h->device));
    h->last_stream = st;
    necg::launch_reset_status(h->d_status, st);  // status = {0, INT_MAX}
    return NECG_OK;
}

int finish_launch() {
    cudaError_t e = cudaGetLastError();
    return cuda_fail(e);
}

// The fused evaluation's launch sequence, from the status reset to the
// partial sums, enqueued on st (no host synchronisation, so it can be captured).
int enqueue_fused(necg_handle *h, LaunchArgs &a, double *f_dev, double *g_dev, size_t siv, cudaStream_t st) {
    necg::launch_reset_status(h->d_status, st);
    mark(h, 0, st);
    if (necg::launch_prep(a, st)) return NECG_ERR_UNSUPPORTED;
    mark(h, 1, st);
    if (necg::launch_fsym(a, st)) return NECG_ERR_ARG;
    if (necg::launch_fsym_tail(a, st)) return NECG_ERR_ARG;
    if (necg::launch_hs_reduce(a, st)) return NECG_ERR_ARG;
    mark(h, 2, st);
    necg::launch_rows_finalize(a, f_dev, g_dev + siv, 0, 0.0, 0.0, st);
    mark(h, 3, st);
    mark(h, 4, st);
    if (necg::launch_fsym_reduce(a, st)) return NECG_ERR_ARG;
    mark(h, 5, st);
    return NECG_OK;
}

// Capture the fused launch sequence on the handle's own stream and keep it as
// the handle's graph for `key`.  On any failure the handle keeps no graph for
// the key and the caller launches eagerly.
void capture_fused(necg_handle *h, LaunchArgs &a, double *f_dev, double *g_dev, size_t siv,
                   const necg_handle::GraphKey &key) {
    if (!h->gstream && cudaStreamCreateWithFlags(&h->gstream, cudaStreamNonBlocking) != cudaSuccess) {
        h->gstream = nullptr;
        cudaGetLastError();
        return;
    }
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(h->gstream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    const int rc = enqueue_fused(h, a, f_dev, g_dev, siv, h->gstream);
    const cudaError_t e = cudaStreamEndCapture(h->gstream, &graph);
    cudaGraphExec_t exec = nullptr;
    const bool ok = rc == NECG_OK && e == cudaSuccess && graph && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    if (!ok) return;
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    h->gexec = exec;
    h->gkey = key;
}

}  // namespace

extern "C" {

int necg_create(int n, int nst, int K_max, double efs, const double *mass_host,
                const double *ncv_host, const double *scvv_host, const double *sml_host,
                const double *sms_host, necg_handle **out) {
    if (!out) return NECG_ERR_ARG;
    *out = nullptr;
    if (n < 1 || n > 6) return NECG_ERR_UNSUPPORTED;
    if (nst < 1 || K_max < 1 || !mass_host || !ncv_host || !scvv_host || !sml_host || !sms_host)
        return NECG_ERR_ARG;
    necg_handle *h = new necg_handle();
    h->n = n;
    h->nst = nst;
    h->K_max = K_max;
    h->efs = efs;
    h->mass.assign(mass_host, mass_host + n * n);
    h->ncv.assign(ncv_host, ncv_host + n + 1);
    h->scvv.assign(scvv_host, scvv_host + nst);
    h->sml.assign(sml_host, sml_host + (size_t)nst * n * n);
    h->sms.assign(sms_host, sms_host + (size_t)nst * 9 * n * n);
    // default tile widths per particle count
    h->lc_e = n >= 5 ? 4 : 8;
    h->lc_g = n >= 5 ? 4 : 8;
    cudaGetDevice(&h->device);
    const size_t K = (size_t)K_max;
    const size_t blk = (size_t)(n * (n + 1) / 2 + 3 * n);
    int rc = NECG_OK;
    if (!rc) rc = dalloc(h, &h->d_sml, h->sml.size());
    if (!rc) rc = dalloc(h, &h->d_sms, h->sms.size());
    if (!rc) rc = dalloc(h, &h->d_scvv, (size_t)nst);
    if (!rc) rc = dalloc(h, &h->d_bra, (size_t)necg::bra_record_size(n) * K);
    if (!rc) rc = dalloc(h, &h->d_ket, (size_t)necg::ket_record_size(n) * K * nst);
    if (!rc) rc = dalloc(h, &h->d_part, (size_t)necg::part_stride(n) * K * ((K + 3) / 4));
    if (!rc) rc = dalloc(h, &h->d_H, K * K);
    if (!rc) rc = dalloc(h, &h->d_S, K * K);
    if (!rc) rc = dalloc(h, &h->d_rows, 2 * K);
    if (!rc) rc = dalloc(h, &h->d_scal, (size_t)4);
    if (!rc) rc = dalloc(h, &h->d_x, K * blk + K);
    if (!rc) rc = dalloc(h, &h->d_g, K * blk + K);
    if (!rc) rc = dalloc(h, &h->d_f, (size_t)2);
    if (!rc) rc = dalloc(h, &h->d_status, (size_t)4);
    cudaStream_t ls = rc ? nullptr : lib_stream(h);
    if (!rc) rc = cuda_fail(cudaMemcpyAsync(h->d_sml, h->sml.data(), h->sml.size() * 8, cudaMemcpyHostToDevice, ls));
    if (!rc) rc = cuda_fail(cudaMemcpyAsync(h->d_sms, h->sms.data(), h->sms.size() * 8, cudaMemcpyHostToDevice, ls));
    if (!rc) rc = cuda_fail(cudaMemcpyAsync(h->d_scvv, h->scvv.data(), h->scvv.size() * 8, cudaMemcpyHostToDevice, ls));
    if (!rc) rc = cuda_fail(cudaMemsetAsync(h->d_status, 0, 16, ls));
    if (!rc) rc = setup_symmetric(h);
    // the workspace is allocated in the library stream's order: make it usable on every stream
    if (!rc) rc = cuda_fail(cudaStreamSynchronize(ls));
    if (rc) {
        free_all(h);
        delete h;
        return rc;
    }
    *out = h;
    return NECG_OK;
}

int necg_destroy(necg_handle *h) {
    if (!h) return NECG_ERR_ARG;
    cudaSetDevice(h->device);
    free_all(h);
    if (h->h_tail) cudaFreeHost(h->h_tail);
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->gstream) cudaStreamDestroy(h->gstream);
    delete h;
    return NECG_OK;
}

long long necg_workspace_bytes(const necg_handle *h) { return h ? h->ws_bytes : -1; }

int necg_set_tiles(necg_handle *h, int lc_energy, int lc_grad) {
    if (!h || lc_energy < 1 || lc_grad < 4 || lc_energy > 4096 || lc_grad > 4096)
        return NECG_ERR_ARG;
    h->lc_e = lc_energy;
    h->lc_g = lc_grad;
    ++h->gversion;
    return NECG_OK;
}

int necg_set_symmetric(necg_handle *h, int mode, int lc, int minw) {
    const bool blockv = minw == 208 || minw == 218 || minw == 228 || minw == 222 || minw == 232 || minw == 248 ||
                        minw == 258 || minw == 268;
    const bool okw = minw == 8 || minw == 12 || minw == 16 ||
                     (mode == 2 && (minw == 108 || minw == 112 || minw == 118 || minw == 122 || blockv));
    if (!h || mode < 0 || mode > 2 || lc < 1 || lc > 64 || !okw) return NECG_ERR_ARG;
    if (blockv && !necg::fused_variant_ok(h->n, minw)) return NECG_ERR_UNSUPPORTED;  // shared memory
    if (mode && !h->sym_ok) return NECG_ERR_UNSUPPORTED;
    h->grad_mode = mode;
    h->lc_s = lc;
    h->minb_s = minw;
    ++h->gversion;
    return NECG_OK;
}

int necg_set_splits(necg_handle *h, int npc) {
    if (!h || npc < 1 || npc > h->nst) return NECG_ERR_ARG;
    h->npc = npc;
    ++h->gversion;
    return NECG_OK;
}

int necg_set_variant(necg_handle *h, int minw_energy, int minw_grad) {
    auto okw = [](int w) { return w == 8 || w == 12 || w == 16 || w == 20; };
    if (!h || !okw(minw_energy) || !(okw(minw_grad) || minw_grad == 112 || minw_grad == 116))
        return NECG_ERR_ARG;
    h->minb_e = minw_energy;
    h->minb_g = minw_grad;
    ++h->gversion;
    return NECG_OK;
}

int necg_build_matrices(necg_handle *h, int K, const double *iv_dev, const double *C_dev,
                        double *H_dev, double *S_dev, double *Kin_dev, double *Pot_dev,
                        double *en_dev, void *stream) {
    int rc = check_K(h, K);
    if (rc) return rc;
    if (!iv_dev) return NECG_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if ((rc = begin(h, st))) return rc;
    if ((rc = ensure_tiles(h, K, st))) return rc;
    LaunchArgs a = base_args(h, K);
    a.iv = iv_dev;
    a.C = C_dev;
    a.H = H_dev ? H_dev : h->d_H;
    a.S = S_dev ? S_dev : h->d_S;
    a.Kin = Kin_dev;
    a.Pot = Pot_dev;
    if (necg::launch_prep(a, st)) return NECG_ERR_UNSUPPORTED;
    necg::launch_energy(a, st);
    if (C_dev && en_dev) necg::launch_rows_finalize(a, nullptr, nullptr, 0, 0.0, 0.0, st, nullptr, en_dev);
    return finish_launch();
}

int necg_outprod(necg_handle *h, int K, const double *x_dev, double *f_dev, double *g_dev,
                 double *H_dev, double *S_dev, void *stream) {
    necg::TraceRange trace("necg_outprod");
    int rc = check_K(h, K);
    if (rc) return rc;
    if (!x_dev || !g_dev) return NECG_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const bool fused = h->grad_mode == 2;
    if (fused) {  // the status reset is part of the fused launch sequence
        CK(cudaSetDevice(h->device));
        h->last_stream = st;
    } else if ((rc = begin(h, st))) {
        return rc;
    }
    if ((rc = ensure_tiles(h, K, st))) return rc;
    const size_t siv = (size_t)K * (h->n * (h->n + 1) / 2 + 3 * h->n);
    LaunchArgs a = base_args(h, K);
    a.iv = x_dev;
    a.C = x_dev + siv;
    a.H = H_dev ? H_dev : h->d_H;
    a.S = S_dev ? S_dev : h->d_S;
    a.g = g_dev;
    if (h->grad_mode >= 1 && (rc = ensure_sym_tiles(h, K, st, h->grad_mode == 2 ? 2 : 1))) return rc;
    if (fused) {
        // fused: one pass over unordered pairs writes H, S and the split gradients
        a.stiles = h->d_stiles;
        a.stile_start = h->d_stile_start;
        a.nstiles = h->nstiles;
        a.LC_s = h->lc_s;
        a.psym = h->d_psym;
        a.sgroups = h->d_sgroups;
        a.nsgroups = h->nsgroups;
        a.qcount = h->d_qcount;
        a.npc = necg::fused_splits(h);
        a.Hp = h->d_Hp;
        a.Sp = h->d_Sp;
        a.xsym = h->d_xsym;
        a.sg_tail0 = h->sg_tail0;
        a.sg_ntail = h->sg_ntail;
        a.sg_parts = h->sg_parts;
        a.urange = h->d_urange;
        // A call that repeats the previous call's buffers, K and settings
        // replays the captured launch sequence (captured the second time the
        // same key is seen, so callers whose buffers change every call stay
        // eager); a stream that is itself being captured gets the launches.
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        CK(cudaStreamIsCapturing(st, &cap));
        const necg_handle::GraphKey key{K, x_dev, f_dev, g_dev, a.H, a.S, h->gversion};
        if (cap == cudaStreamCaptureStatusNone) {
            if (!(h->gexec && h->gkey == key) && h->gseen == key) capture_fused(h, a, f_dev, g_dev, siv, key);
            if (h->gexec && h->gkey == key) {
                CK(cudaGraphLaunch(h->gexec, st));
                return finish_launch();
            }
        }
        h->gseen = key;
        if ((rc = enqueue_fused(h, a, f_dev, g_dev, siv, st))) return rc;
        return finish_launch();
    }
    mark(h, 0, st);
    if (necg::launch_prep(a, st)) return NECG_ERR_UNSUPPORTED;
    mark(h, 1, st);
    necg::launch_energy(a, st);
    mark(h, 2, st);
    necg::launch_rows_finalize(a, f_dev, g_dev + siv, 0, 0.0, 0.0, st);
    if ((rc = launch_gradient(h, a, st))) return rc;
    return finish_launch();
}

// ---- one evaluation split across ranks (tiles of the fused pass) -----------
namespace {
int shard_args(necg_handle *h, int K, const double *x_dev, int t0, int t1, cudaStream_t st, LaunchArgs &a) {
    int rc = check_K(h, K);
    if (rc) return rc;
    if (!x_dev) return NECG_ERR_ARG;
    if (!h->sym_ok) return NECG_ERR_UNSUPPORTED;
    CK(cudaSetDevice(h->device));
    if ((rc = ensure_sym_tiles(h, K, st, 2))) return rc;
    if (t0 < 0 || t1 < t0 || t1 > h->nstiles) return NECG_ERR_ARG;
    a = base_args(h, K);
    const size_t siv = (size_t)K * (h->n * (h->n + 1) / 2 + 3 * h->n);
    a.iv = x_dev;
    a.C = x_dev + siv;
    a.H = h->d_H;
    a.S = h->d_S;
    a.stiles = h->d_stiles;
    a.stile_start = h->d_stile_start;
    a.nstiles = h->nstiles;
    a.LC_s = h->lc_s;
    a.psym = h->d_psym;
    a.st_begin = t0;
    a.st_end = t1;
    return NECG_OK;
}
}  // namespace

int necg_shard_tiles(necg_handle *h, int K, int *ntiles) {
    if (!ntiles) return NECG_ERR_ARG;
    int rc = check_K(h, K);
    if (rc) return rc;
    if (!h->sym_ok) return NECG_ERR_UNSUPPORTED;
    CK(cudaSetDevice(h->device));
    if ((rc = ensure_sym_tiles(h, K, h->last_stream, 2))) return rc;
    *ntiles = h->nstiles;
    return NECG_OK;
}

int necg_shard_pairs(necg_handle *h, int K, const double *x_dev, int tile_begin, int tile_end,
                     double *rows_dev, void *stream) {
    necg::TraceRange trace("necg_shard_pairs");
    cudaStream_t st = (cudaStream_t)stream;
    LaunchArgs a;
    int rc = shard_args(h, K, x_dev, tile_begin, tile_end, st, a);
    if (rc) return rc;
    if (!rows_dev) return NECG_ERR_ARG;
    if ((rc = begin(h, st))) return rc;
    // this shard writes only its tiles' entries of H and S: the rest must be 0
    CK(cudaMemsetAsync(h->d_H, 0, sizeof(double) * (size_t)K * K, st));
    CK(cudaMemsetAsync(h->d_S, 0, sizeof(double) * (size_t)K * K, st));
    if (necg::launch_prep(a, st)) return NECG_ERR_UNSUPPORTED;
    if (tile_end > tile_begin && necg::launch_fsym(a, st)) return NECG_ERR_ARG;
    if (necg::launch_rows(a, rows_dev, st)) return NECG_ERR_ARG;
    return finish_launch();
}

int necg_shard_grad(necg_handle *h, int K, const double *x_dev, const double *rows_dev, int tile_begin,
                    int tile_end, double *f_dev, double *g_dev, double *sums_dev, void *stream) {
    necg::TraceRange trace("necg_shard_grad");
    cudaStream_t st = (cudaStream_t)stream;
    LaunchArgs a;
    int rc = shard_args(h, K, x_dev, tile_begin, tile_end, st, a);
    if (rc) return rc;
    if (!rows_dev || !g_dev || !sums_dev) return NECG_ERR_ARG;
    h->last_stream = st;
    const size_t siv = (size_t)K * (h->n * (h->n + 1) / 2 + 3 * h->n);
    a.g = g_dev;
    a.sums = sums_dev;
    necg::launch_finalize(a, rows_dev, f_dev, g_dev + siv, st);
    if (necg::launch_fsym_reduce(a, st)) return NECG_ERR_ARG;  // per-basis sums of this shard's tiles only
    return finish_launch();
}

int necg_shard_finish(necg_handle *h, int K, const double *x_dev, const double *sums_dev, double *g_dev,
                      void *stream) {
    necg::TraceRange trace("necg_shard_finish");
    int rc = check_K(h, K);
    if (rc) return rc;
    if (!x_dev || !sums_dev || !g_dev) return NECG_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    CK(cudaSetDevice(h->device));
    h->last_stream = st;
    LaunchArgs a = base_args(h, K);
    const size_t siv = (size_t)K * (h->n * (h->n + 1) / 2 + 3 * h->n);
    a.iv = x_dev;
    a.C = x_dev + siv;
    a.g = g_dev;
    if (necg::launch_reduce_sums(a, sums_dev, st)) return NECG_ERR_ARG;
    return finish_launch();
}

int necg_outprod_host(necg_handle *h, int K, const double *x_host, double *f_host,
                      double *g_host, void *stream) {
    necg::TraceRange trace("necg_outprod_host");
    int rc = check_K(h, K);
    if (rc) return rc;
    if (!x_host || !g_host) return NECG_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    CK(cudaSetDevice(h->device));
    const size_t len = (size_t)K * (h->n * (h->n + 1) / 2 + 3 * h->n) + K;
    CK(cudaMemcpyAsync(h->d_x, x_host, len * sizeof(double), cudaMemcpyHostToDevice, st));
    rc = necg_outprod(h, K, h->d_x, h->d_f, h->d_g, nullptr, nullptr, stream);
    if (rc) return rc;
    // f and the status words land in a pinned buffer, so the stream is waited for once
    if (!h->h_tail) CK(cudaMallocHost((void **)&h->h_tail, 4 * sizeof(double)));
    CK(cudaMemcpyAsync(g_host, h->d_g, len * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(h->h_tail, h->d_f, sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(h->h_tail + 1, h->d_status, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (f_host) *f_host = h->h_tail[0];
    int sw[2];
    memcpy(sw, h->h_tail + 1, sizeof(sw));
    return status_code(sw, nullptr);
}

int necg_make_grad(necg_handle *h, int K, const double *iv_dev, const double *C_dev,
                   const double *H_dev, const double *S_dev, double eng, double norm,
                   double *g_dev, void *stream) {
    necg::TraceRange trace("necg_make_grad");
    int rc = check_K(h, K);
    if (rc) return rc;
    if (!iv_dev || !C_dev || !H_dev || !S_dev || !g_dev) return NECG_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if ((rc = begin(h, st))) return rc;
    const size_t siv = (size_t)K * (h->n * (h->n + 1) / 2 + 3 * h->n);
    LaunchArgs a = base_args(h, K);
    a.iv = iv_dev;
    a.C = C_dev;
    a.H = const_cast<double *>(H_dev);
    a.S = const_cast<double *>(S_dev);
    a.g = g_dev;
    if (necg::launch_prep(a, st)) return NECG_ERR_UNSUPPORTED;
    // GRADC = 2 norm (H - eng S) C with the caller's eng and norm; also sets
    // the E and norm the gradient tiles read
    necg::launch_rows_finalize(a, nullptr, g_dev + siv, 1, eng, norm, st);
    if ((rc = launch_gradient(h, a, st))) return rc;
    return finish_launch();
}

int necg_make_grad_dev(necg_handle *h, int K, const double *iv_dev, const double *C_dev,
                       const double *H_dev, const double *S_dev, const double *en_dev, double *g_dev,
                       void *stream) {
    int rc = check_K(h, K);
    if (rc) return rc;
    if (!iv_dev || !C_dev || !H_dev || !S_dev || !en_dev || !g_dev) return NECG_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if ((rc = begin(h, st))) return rc;
    const size_t siv = (size_t)K * (h->n * (h->n + 1) / 2 + 3 * h->n);
    LaunchArgs a = base_args(h, K);
    a.iv = iv_dev;
    a.C = C_dev;
    a.H = const_cast<double *>(H_dev);
    a.S = const_cast<double *>(S_dev);
    a.g = g_dev;
    if (necg::launch_prep(a, st)) return NECG_ERR_UNSUPPORTED;
    necg::launch_rows_finalize(a, nullptr, g_dev + siv, 2, 0.0, 0.0, st, en_dev, nullptr);
    if ((rc = launch_gradient(h, a, st))) return rc;
    return finish_launch();
}

int necg_matel(necg_handle *h, int K, const double *iv_dev, int nterms, const int *terms_dev,
               double *out_dev, void *stream) {
    int rc = check_K(h, K);
    if (rc) return rc;
    if (!iv_dev || nterms < 0 || (nterms > 0 && (!terms_dev || !out_dev))) return NECG_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if ((rc = begin(h, st))) return rc;
    LaunchArgs a = base_args(h, K);
    a.iv = iv_dev;
    a.C = nullptr;
    if (necg::launch_prep(a, st)) return NECG_ERR_UNSUPPORTED;
    if (nterms > 0) necg::launch_matel(a, terms_dev, nterms, out_dev, st);
    return finish_launch();
}

int necg_rrms(necg_handle *h, int K, const double *iv_dev, int nterms, const int *terms_dev,
              double *out_dev, void *stream) {
    int rc = check_K(h, K);
    if (rc) return rc;
    if (!iv_dev || nterms < 0 || (nterms > 0 && (!terms_dev || !out_dev))) return NECG_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if ((rc = begin(h, st))) return rc;
    LaunchArgs a = base_args(h, K);
    a.iv = iv_dev;
    a.C = nullptr;
    if (necg::launch_prep(a, st)) return NECG_ERR_UNSUPPORTED;
    if (nterms > 0) necg::launch_rrms(a, terms_dev, nterms, out_dev, st);
    return finish_launch();
}

int necg_dipole(necg_handle *h, int K, const double *iv_dev, const double *C_dev, double *comps_dev,
                double *dipole_dev, void *stream) {
    int rc = check_K(h, K);
    if (rc) return rc;
    if (!iv_dev || !C_dev || !comps_dev) return NECG_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if ((rc = begin(h, st))) return rc;
    if ((rc = ensure_tiles(h, K, st))) return rc;
    LaunchArgs a = base_args(h, K);
    // the tile partials reuse the gradient-partial workspace
    const size_t need = (size_t)a.ntiles * (3 * h->n + 1);
    const size_t cap = (size_t)necg::part_stride(h->n) * h->K_max * ((h->K_max + 3) / 4);
    if (need > cap) return NECG_ERR_CAPACITY;
    a.iv = iv_dev;
    a.C = C_dev;
    if (necg::launch_prep(a, st)) return NECG_ERR_UNSUPPORTED;
    necg::launch_dipole(a, h->d_part, comps_dev, dipole_dev, st);
    return finish_launch();
}

int necg_gradel(necg_handle *h, int K, const double *iv_dev, int nterms, const int *terms_dev,
                double *tgvl_dev, double *tgvls_dev, void *stream) {
    int rc = check_K(h, K);
    if (rc) return rc;
    if (!iv_dev || nterms < 0 || (nterms > 0 && (!terms_dev || !tgvl_dev || !tgvls_dev)))
        return NECG_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if ((rc = begin(h, st))) return rc;
    LaunchArgs a = base_args(h, K);
    a.iv = iv_dev;
    a.C = nullptr;
    if (necg::launch_prep(a, st)) return NECG_ERR_UNSUPPORTED;
    if (nterms > 0) necg::launch_gradel(a, terms_dev, nterms, tgvl_dev, tgvls_dev, st);
    return finish_launch();
}

int necg_f0(const double *z_dev, int count, double *f_dev, double *df_dev, void *stream) {
    if (count < 0 || (count > 0 && !z_dev)) return NECG_ERR_ARG;
    if (count == 0) return NECG_OK;
    necg::launch_f0(z_dev, count, f_dev, df_dev, (cudaStream_t)stream);
    return finish_launch();
}

int necg_status(necg_handle *h, long long *bad_pair) {
    if (!h) return NECG_ERR_ARG;
    CK(cudaSetDevice(h->device));
    int st[2];
    CK(cudaMemcpyAsync(st, h->d_status, sizeof(st), cudaMemcpyDeviceToHost, h->last_stream));
    CK(cudaStreamSynchronize(h->last_stream));
    return status_code(st, bad_pair);
}

int necg_profile(necg_handle *h, int enable) {
    if (!h) return NECG_ERR_ARG;
    CK(cudaSetDevice(h->device));
    if (enable && !h->ev[0])
        for (cudaEvent_t &e : h->ev) CK(cudaEventCreate(&e));
    h->profile = enable != 0;
    ++h->gversion;
    return NECG_OK;
}

int necg_phase_ms(necg_handle *h, double *ms) {
    if (!h || !ms || !h->ev[0]) return NECG_ERR_ARG;
    CK(cudaSetDevice(h->device));
    CK(cudaEventSynchronize(h->ev[5]));
    for (int i = 0; i < 5; ++i) {
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, h->ev[i], h->ev[i + 1]));
        ms[i] = t;
    }
    return NECG_OK;
}

int necg_fp64_peak(int iters, double *tflops, void *stream) {
    if (iters < 1 || !tflops) return NECG_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0, sms = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = sms * 8;
    double *sink = nullptr;
    CK(cudaMalloc((void **)&sink, blocks * sizeof(double)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    necg::launch_fp64_probe(blocks, iters / 4 + 1, sink, st);  // warm-up
    cudaEventRecord(e0, st);
    necg::launch_fp64_probe(blocks, iters, sink, st);
    cudaEventRecord(e1, st);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (e != cudaSuccess) return cuda_fail(e);
    const double flops = 2.0 * 8.0 * (double)iters * blocks * 256.0;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return NECG_OK;
}

const char *necg_status_string(int code) {
    switch (code) {
    case NECG_OK: return "ok";
    case NECG_ERR_ARG: return "invalid argument";
    case NECG_ERR_NOT_PD: return "A_k + A_l' is not positive definite for some basis pair";
    case NECG_ERR_NONFINITE: return "non-finite energy or gradient";
    case NECG_ERR_CUDA: return "CUDA runtime error";
    case NECG_ERR_ALLOC: return "device allocation failed";
    case NECG_ERR_UNSUPPORTED: return "unsupported particle count (1..6)";
    case NECG_ERR_CAPACITY: return "K exceeds the handle's K_max";
    default: return "unknown status";
    }
}

}  // extern "C"
