// necg_kernels.cuh -- launcher interface between the C-ABI layer and the kernels.
#pragma once
#include <cuda_runtime.h>

#include "necg_lanes.cuh"

namespace necg {

struct LaunchArgs {
    int n, K, nst;
    double efs;
    const double *mass_h, *ncv_h;          // host copies (folded into kernel constants)
    const double *iv, *C;                  // device: packed parameters, coefficients
    const double *sml, *sms, *scvv;        // device: symmetry set
    double *bra, *ket;                     // device workspace: bra SoA, ket records
    const int2 *tiles;                     // energy tile list (kb, lc)
    int ntiles, LC_e, LC_g;
    int minb_e, minb_g;                    // kernel variants: min resident blocks per SM
    double *H, *S, *Kin, *Pot;             // device outputs (Kin/Pot optional)
    double *rows, *scal, *part, *g;        // device workspace / outputs
    double lam, scale_override;
    int *status;
    // symmetric gradient pass
    const int *pinv;                       // index of P^-1 per symmetry term (null: none)
    KetMap kmap;                           // ket frame map per (P, field)
    const int2 *stiles;                    // lower-triangle tiles of chunk LC_s
    const int *stile_start;                // first tile of each 32-row block (nkb + 1)
    int nstiles, LC_s, minb_s;
    double *psym;                          // bra partials, then ket partials
    // shard of the fused pass: tiles [st_begin, st_end) (st_end = 0: all);
    // sums (non-null): write the per-basis sums there and stop before GRADA
    int st_begin, st_end;
    double *sums;
    // block-synchronised fused pass (variant 208): groups of 8 tiles of one row block
    const int2 *sgroups;                   // (kb, first lc)
    int nsgroups;
    int *qcount;                           // group queue head (reset before the launch)
    // fused pass with the symmetry terms split over npc tiles per (kb, lc) (one-warp
    // variants; npc <= 1: no split): split pc writes its H, S sums to Hp, Sp + pc K^2
    int npc;
    double *Hp, *Sp;
    // lockstep pass: the last sg_ntail groups of the queue are split into
    // sg_parts units over the symmetry terms, from queue index sg_tail0; parts
    // 1 .. sg_parts - 1 write to xsym (fsym_tail_slot doubles per tile and part)
    double *xsym;
    int sg_tail0, sg_ntail, sg_parts;
    // lockstep pass: bra partials are written per queue unit; row block kb's
    // units are [urange[kb].x, urange[kb].y)
    const int2 *urange;
};

// A tile group of the lockstep pass: row block kb, first ket chunk lc0 and, for
// a split group of the queue's tail, its part and the number of parts (one part
// per range of symmetry terms).
__host__ __device__ inline int2 sgroup_pack(int kb, int lc0, int part, int parts) {
    return make_int2(kb, lc0 | (part << 20) | (parts << 24));
}
__host__ __device__ inline int sgroup_lc0(int2 g) { return g.y & 0xFFFFF; }
__host__ __device__ inline int sgroup_part(int2 g) { return (g.y >> 20) & 0xF; }
__host__ __device__ inline int sgroup_parts(int2 g) { return ((g.y >> 24) & 0xF) > 1 ? ((g.y >> 24) & 0xF) : 1; }


int launch_prep(const LaunchArgs &a, cudaStream_t st);
int launch_energy(const LaunchArgs &a, cudaStream_t st);
int launch_grad(const LaunchArgs &a, cudaStream_t st);
int launch_gsym(const LaunchArgs &a, cudaStream_t st);
int launch_gsym_reduce(const LaunchArgs &a, cudaStream_t st);
// fused energy + symmetric gradient pass (writes H, S and split partials) and
// its reduction (needs E in scal, i.e. after launch_rows_finalize)
int launch_fsym(const LaunchArgs &a, cudaStream_t st);
// lockstep-block variants of the fused pass (2xy): warps per block, and
// whether the variant's shared memory fits for n particles
int fused_block_warps(int variant);
bool fused_variant_ok(int n, int variant);
int launch_fsym_reduce(const LaunchArgs &a, cudaStream_t st);
// H, S = sum over the splits of Hp, Sp (fused pass with npc > 1), before rows/finalize
int launch_hs_reduce(const LaunchArgs &a, cudaStream_t st);
// add the split parts of the lockstep pass's tail tiles into the main buffers
// (after launch_fsym, before H and S are read)
int launch_fsym_tail(const LaunchArgs &a, cudaStream_t st);
int launch_grad_tiles(const LaunchArgs &a, cudaStream_t st);
int launch_grad_reduce(const LaunchArgs &a, cudaStream_t st);
int launch_matel(const LaunchArgs &a, const int *terms, int nterms, double *out, cudaStream_t st);
// dipole: per-term rrms elements, and the C-contracted sums over the energy
// tiles (part: ntiles * (3n + 1) doubles) reduced into comps[3n] and dip[3]
int launch_rrms(const LaunchArgs &a, const int *terms, int nterms, double *out, cudaStream_t st);
int launch_dipole(const LaunchArgs &a, double *part, double *comps, double *dip, cudaStream_t st);
int launch_gradel(const LaunchArgs &a, const int *terms, int nterms, double *tg, double *tgs,
                  cudaStream_t st);
// given: 0 compute E and norm from C, H, S; 1 use (eng, norm); 2 read them
// from given_dev[0..1].  en_out (optional) receives {E, norm}.
void launch_rows_finalize(const LaunchArgs &a, double *f_out, double *gradc, int given,
                          double eng, double norm, cudaStream_t st,
                          const double *given_dev = nullptr, double *en_out = nullptr);
void launch_reset_status(int *status, cudaStream_t st);
// pieces of a sharded evaluation: rows (H C, S C) of this shard's H and S;
// E, norm and GRADC from given rows; GRADA from given per-basis sums
int launch_rows(const LaunchArgs &a, double *rows, cudaStream_t st);
void launch_finalize(const LaunchArgs &a, const double *rows, double *f_out, double *gradc, cudaStream_t st);
int launch_reduce_sums(const LaunchArgs &a, const double *sums, cudaStream_t st);
void launch_fp64_probe(int blocks, int iters, double *sink, cudaStream_t st);
void launch_f0(const double *z, int count, double *f, double *df, cudaStream_t st);

// sizes in doubles
int ket_record_size(int n);
int bra_record_size(int n);
int part_stride(int n);

}  // namespace necg
