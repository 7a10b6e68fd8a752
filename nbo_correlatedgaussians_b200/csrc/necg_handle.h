// necg_handle.h -- internal layout of the opaque necg_handle (one particle
// system + symmetry set + device workspace for bases of up to K_max functions).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "../../include/necg.h"

struct necg_handle {
    int n, nst, K_max;
    double efs;
    std::vector<double> mass, ncv, scvv, sml, sms;
    double *d_sml = nullptr, *d_sms = nullptr, *d_scvv = nullptr;
    double *d_bra = nullptr, *d_ket = nullptr, *d_part = nullptr;
    double *d_H = nullptr, *d_S = nullptr, *d_rows = nullptr, *d_scal = nullptr;
    double *d_x = nullptr, *d_g = nullptr, *d_f = nullptr;
    int *d_status = nullptr;
    int2 *d_tiles = nullptr;
    int tiles_cap = 0, tiles_K = -1, tiles_lc = -1, ntiles = 0;
    int lc_e = 8, lc_g = 8;
    int minb_e = 16, minb_g = 8;
    int device = 0;
    cudaStream_t last_stream = nullptr;
    long long ws_bytes = 0;
    bool profile = false;
    cudaEvent_t ev[6] = {};
    // symmetric gradient pass (when the symmetry set is closed under inverse)
    bool sym_ok = false;
    int grad_mode = 0;  // 0 ordered pairs, 1 symmetric, 2 fused energy + symmetric
    int lc_s = 4, minb_s = 8;
    int *d_pinv = nullptr;
    int *d_kcnt = nullptr, *d_ksrc = nullptr;
    double *d_kcoef = nullptr;
    int kmaxnz = 0;
    int2 *d_stiles = nullptr;
    int *d_stile_start = nullptr;
    int stiles_cap = 0, stiles_K = -1, stiles_lc = -1, nstiles = 0;
    double *d_psym = nullptr;
    size_t psym_cap = 0;  // doubles
    int2 *d_sgroups = nullptr;  // groups of 8 fused tiles of one row block (kb, first lc)
    int sgroups_cap = 0, nsgroups = 0, sgroups_w = 0;
    // the queue's tail: its last sg_ntail groups split into sg_parts units from
    // queue index sg_tail0; parts after the first write to d_xsym
    int sg_tail0 = 0, sg_ntail = 0, sg_parts = 1;
    double *d_xsym = nullptr;
    size_t xsym_cap = 0;  // doubles
    int2 *d_urange = nullptr;  // queue units of each row block (bra partial slots)
    int urange_cap = 0;
    int *d_qcount = nullptr;    // queue head of the block-synchronised fused pass
    int2 *d_bgroups = nullptr;  // the same groups with 8 chunks each (the batched step's blocks)
    int bgroups_cap = 0, nbgroups = 0;
    // fused pass with one-warp tiles: symmetry terms split over npc warps per tile
    int npc = 1;
    double *d_Hp = nullptr, *d_Sp = nullptr;  // npc K x K sums each
    size_t hp_cap = 0;                        // doubles per buffer
    // pinned host landing area of the host entry point: f, then the two status words
    double *h_tail = nullptr;
    // the fused evaluation's launch sequence as a CUDA graph: captured (on the
    // handle's own stream) the second time a call repeats the same key, then
    // replayed on the caller's stream while the key stays the same
    struct GraphKey {
        int K = -1;
        const void *x = nullptr, *f = nullptr, *g = nullptr, *H = nullptr, *S = nullptr;
        int version = -1;
        bool operator==(const GraphKey &o) const {
            return K == o.K && x == o.x && f == o.f && g == o.g && H == o.H && S == o.S && version == o.version;
        }
    };
    int gversion = 0;  // bumped by every change of settings, tiles or buffers
    GraphKey gkey, gseen;
    cudaGraphExec_t gexec = nullptr;
    cudaStream_t gstream = nullptr;
};

namespace necg {
// Tile list and partial buffers of the fused pass for bases of K functions
// (the handle's ket chunk lc_s), as the batched step needs them; returns a
// status code.  May synchronise `st` when the list changes.
int prepare_fused(necg_handle *h, int K, cudaStream_t st);
// Splits of the symmetry terms per one-warp tile of the fused pass (1: none):
// npc when the handle runs the fused pass with a one-warp variant, else 1.
inline int fused_splits(const necg_handle *h) {
    return h->grad_mode == 2 && h->minb_s < 200 && h->npc > 1 ? h->npc : 1;
}
}  // namespace necg
