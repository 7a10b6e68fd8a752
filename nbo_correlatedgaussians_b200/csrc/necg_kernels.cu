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
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "necg_math.cuh"
#include "necg_kernels.cuh"

namespace necg {

// ---------------------------------------------------------------------------
// Status word: [0] bit flags, [1] first failing pair (row-major k*K + l).
__device__ __forceinline__ void flag_bad_pair(int *status, int flag, int pair) {
    atomicOr(status, flag);
    atomicMin(status + 1, pair);
}

// Unpack vech(L) (python/matel.py:59-66: column-major lower triangle) into a
// packed-lower row-major array.
template <int N>
__device__ __forceinline__ void unpack_L(const double *blk, double (&L)[tri(N)]) {
    int idx = 0;
#pragma unroll
    for (int j = 0; j < N; ++j)
#pragma unroll
        for (int i = j; i < N; ++i) L[sx(i, j)] = blk[idx++];
}

// A = L L^T (packed)
template <int N>
__device__ __forceinline__ void llt(const double (&L)[tri(N)], double (&A)[tri(N)]) {
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k <= j; ++k) s += L[sx(i, k)] * L[sx(j, k)];
            A[sx(i, j)] = s;
        }
}

// A M A (packed), A M (full) and tr(M A)
template <int N>
__device__ __forceinline__ void mass_products(const double (&A)[tri(N)], const double *M,
                                              double (&AM)[N * N], double (&AMA)[tri(N)],
                                              double &tMA) {
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < N; ++k) s += A[sx(i, k)] * M[k * N + j];
            AM[i * N + j] = s;
        }
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < N; ++k) s += AM[i * N + k] * A[sx(k, j)];
            AMA[sx(i, j)] = s;
        }
    double t = 0.0;
#pragma unroll
    for (int i = 0; i < N; ++i) t += AM[i * N + i];
    tMA = t;
}

template <int N>
__global__ void __launch_bounds__(128) prep_bra_kernel(const double *__restrict__ iv, int K,
                                                       Consts<N> cs, double *__restrict__ bra) {
    using BL = BraLayout<N>;
    constexpr int blk = tri(N) + 3 * N;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    const double *b = iv + (size_t)k * blk;
    double L[tri(N)], A[tri(N)], S[3 * N], AS[3 * N], AM[N * N], AMA[tri(N)], tMA;
    unpack_L<N>(b, L);
#pragma unroll
    for (int t = 0; t < 3 * N; ++t) S[t] = b[tri(N) + t];
    llt<N>(L, A);
    symv3<N>(A, 0, S, AS);
    mass_products<N>(A, cs.M, AM, AMA, tMA);
    double i1 = 0.0, dl = 1.0;
#pragma unroll
    for (int t = 0; t < 3 * N; ++t) i1 += S[t] * AS[t];
#pragma unroll
    for (int i = 0; i < N; ++i) dl *= L[sx(i, i)];
    dl = fabs(dl);
    const size_t KK = (size_t)K;
#pragma unroll
    for (int t = 0; t < tri(N); ++t) bra[(BL::A + t) * KK + k] = A[t];
#pragma unroll
    for (int t = 0; t < 3 * N; ++t) bra[(BL::S + t) * KK + k] = S[t];
#pragma unroll
    for (int t = 0; t < 3 * N; ++t) bra[(BL::AS + t) * KK + k] = AS[t];
#pragma unroll
    for (int t = 0; t < tri(N); ++t) bra[(BL::Nk + t) * KK + k] = AMA[t];
    bra[BL::i1 * KK + k] = i1;
    bra[BL::pre * KK + k] = dl * sqrt(dl);
    bra[BL::tMA * KK + k] = tMA;
#pragma unroll
    for (int t = 0; t < tri(N); ++t) bra[(BL::L + t) * KK + k] = L[t];
}

// Ket records: python/matel.py:76-87 (al <- sml^T al sml, st2 <- sms st2)
template <int N>
__global__ void __launch_bounds__(128) prep_ket_kernel(const double *__restrict__ iv,
                                                       const double *__restrict__ C, int K,
                                                       int nst, Consts<N> cs,
                                                       const double *__restrict__ sml,
                                                       const double *__restrict__ sms,
                                                       const double *__restrict__ scvv,
                                                       double *__restrict__ ket) {
    using KL = KetLayout<N>;
    constexpr int blk = tri(N) + 3 * N;
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= K * nst) return;
    const int l = id / nst, P = id - l * nst;
    const double *b = iv + (size_t)l * blk;
    double L[tri(N)], A[tri(N)];
    unpack_L<N>(b, L);
    llt<N>(L, A);
    const double *pm = sml + (size_t)P * N * N;
    // Ap = pm^T A pm
    double Apm[N * N];
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < N; ++k) s += A[sx(i, k)] * pm[k * N + j];
            Apm[i * N + j] = s;
        }
    double Ap[tri(N)];
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < N; ++k) s += pm[k * N + i] * Apm[k * N + j];
            Ap[sx(i, j)] = s;
        }
    // Sp = sms[P] s_l (3n x 3n general map)
    const double *sm = sms + (size_t)P * 9 * N * N;
    double Sp[3 * N];
#pragma unroll
    for (int r = 0; r < 3 * N; ++r) {
        double s = 0.0;
#pragma unroll
        for (int c = 0; c < 3 * N; ++c) s += sm[r * 3 * N + c] * b[tri(N) + c];
        Sp[r] = s;
    }
    double ASp[3 * N], AM[N * N], AMA[tri(N)], tMA;
    symv3<N>(Ap, 0, Sp, ASp);
    mass_products<N>(Ap, cs.M, AM, AMA, tMA);
    double i2 = 0.0, dl = 1.0;
#pragma unroll
    for (int t = 0; t < 3 * N; ++t) i2 += Sp[t] * ASp[t];
#pragma unroll
    for (int i = 0; i < N; ++i) dl *= L[sx(i, i)];
    dl = fabs(dl);
    double *o = ket + (size_t)id * KL::size;
#pragma unroll
    for (int t = 0; t < tri(N); ++t) o[KL::Ap + t] = Ap[t];
#pragma unroll
    for (int t = 0; t < 3 * N; ++t) o[KL::Sp + t] = Sp[t];
#pragma unroll
    for (int t = 0; t < 3 * N; ++t) o[KL::ASp + t] = ASp[t];
#pragma unroll
    for (int t = 0; t < tri(N); ++t) o[KL::Np + t] = AMA[t];
#pragma unroll
    for (int t = 0; t < N * N; ++t) o[KL::AMp + t] = AM[t];
    o[KL::i2] = i2;
    o[KL::pre] = dl * sqrt(dl);
    o[KL::tMA] = tMA;
    o[KL::w] = scvv[P];
    o[KL::wC] = C ? 2.0 * scvv[P] * C[l] : 0.0;
    if (KL::size > KL::wC + 1) o[KL::wC + 1] = 0.0;
}

// ---------------------------------------------------------------------------
// Energy tiles over the lower triangle (the loop of python/outprod.py:49-54 and
// python/necg.py:43-50).  Tile t covers bra k in [32 kb, 32 kb + 32) and ket
// l in [lc LC, lc LC + LC) with l <= k.  Kin / Pot may be null.
template <int N>
__global__ void __launch_bounds__(128) energy_kernel(const int2 *__restrict__ tiles, int ntiles,
                                                     int LC, int K, int nst, Consts<N> cs,
                                                     const double *__restrict__ bra,
                                                     const double *__restrict__ ket,
                                                     double *__restrict__ H, double *__restrict__ S,
                                                     double *__restrict__ Kin,
                                                     double *__restrict__ Pot, int *status) {
    using KL = KetLayout<N>;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= ntiles) return;
    const int2 tl = tiles[warp];
    const int k = tl.x * 32 + lane;
    const int l0 = tl.y * LC;
    const int l1 = min(l0 + LC, K);
    if (k >= K || l0 > k) return;
    const BraRef b{bra + k, (size_t)K};
    const int lend = min(l1, k + 1);
    for (int l = l0; l < lend; ++l) {
        double h = 0.0, s = 0.0, tkin = 0.0, tpot = 0.0;
        bool ok = true;
        const double *kr = ket + (size_t)l * nst * KL::size;
        for (int P = 0; P < nst; ++P, kr += KL::size) {
            double ov, tau, rho, sig;
            ok = term_energy<N>(b, kr, cs, ov, tau, rho, sig) && ok;
            const double w = kr[KL::w];
            h += w * ov * (2.0 * tau + rho - sig);
            s += w * ov;
            tkin += w * ov * 2.0 * tau;
            tpot += w * ov * rho;
        }
        if (!ok) flag_bad_pair(status, 1, k * K + l);
        if (!isfinite(h) || !isfinite(s)) flag_bad_pair(status, 2, k * K + l);
        H[(size_t)k * K + l] = h;
        H[(size_t)l * K + k] = h;
        S[(size_t)k * K + l] = s;
        S[(size_t)l * K + k] = s;
        if (Kin) {
            Kin[(size_t)k * K + l] = tkin;
            Kin[(size_t)l * K + k] = tkin;
        }
        if (Pot) {
            Pot[(size_t)k * K + l] = tpot;
            Pot[(size_t)l * K + k] = tpot;
        }
    }
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
// GRADC = 2 norm (H - E S) C (python/make_grad.py:85) into g[siv .. siv+K).
// scal = {E, norm, cHc, cSc}.  With `given`, E and norm are the caller's
// (make_grad(eng, norm) semantics).  One block of 1024 threads; fixed-order tree.
__global__ void __launch_bounds__(1024) finalize_kernel(const double *__restrict__ rows,
                                                        const double *__restrict__ C, int K,
                                                        double *__restrict__ scal,
                                                        double *__restrict__ f_out,
                                                        double *__restrict__ gradc,
                                                        int *status, int given, double eng,
                                                        double gnorm) {
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
            const double E = given ? eng : ah / as;
            const double nrm = given ? gnorm : 1.0 / as;
            scal[0] = E;
            scal[1] = nrm;
            scal[2] = ah;
            scal[3] = as;
            if (f_out) *f_out = E;
            if (!isfinite(E)) atomicOr(status, 2);
            sh[0][0] = E;
            sh[1][0] = nrm;
        }
    }
    __syncthreads();
    const double E = sh[0][0], norm = sh[1][0];
    if (gradc)
        for (int i = threadIdx.x; i < K; i += blockDim.x)
            gradc[i] = 2.0 * norm * (rows[i] - E * rows[K + i]);
}

// ---------------------------------------------------------------------------
// Gradient tiles over the full square of ordered pairs (the loop of
// python/make_grad.py:37-55 contracted with C on the fly, lines 61-79).
// Tile t = (kb, lc); lane k accumulates, over l in the chunk and all P,
//   wC(l,P) * d/d(A_k, s_k) [lam h - E ov]
// and writes its partial to part[(lc * PS + f) * K + k].
template <int N>
__global__ void __launch_bounds__(128) grad_kernel(int nkb, int nlc, int LC, int K, int nst,
                                                   Consts<N> cs, const double *__restrict__ bra,
                                                   const double *__restrict__ ket,
                                                   const double *__restrict__ scal, double lam,
                                                   double *__restrict__ part, int *status) {
    using KL = KetLayout<N>;
    constexpr int PS = tri(N) + 1 + 3 * N;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nkb * nlc) return;
    const int kb = warp % nkb, lc = warp / nkb;
    const int k = kb * 32 + lane;
    if (k >= K) return;
    const int l0 = lc * LC, l1 = min(l0 + LC, K);
    const double E = scal[0];
    const BraRef b{bra + k, (size_t)K};
    double accG[tri(N)], accS[3 * N], accD = 0.0;
#pragma unroll
    for (int t = 0; t < tri(N); ++t) accG[t] = 0.0;
#pragma unroll
    for (int t = 0; t < 3 * N; ++t) accS[t] = 0.0;
    bool ok = true;
    for (int l = l0; l < l1; ++l) {
        const double *kr = ket + (size_t)l * nst * KL::size;
        for (int P = 0; P < nst; ++P, kr += KL::size)
            ok = term_grad<N>(b, kr, cs, lam, E, kr[KL::wC], accG, accD, accS) && ok;
    }
    if (!ok) flag_bad_pair(status, 1, k * K + l0);
    double *o = part + (size_t)lc * PS * K + k;
#pragma unroll
    for (int t = 0; t < tri(N); ++t) o[(size_t)t * K] = accG[t];
    o[(size_t)tri(N) * K] = accD;
#pragma unroll
    for (int t = 0; t < 3 * N; ++t) o[(size_t)(tri(N) + 1 + t) * K] = accS[t];
}

// Sum the nlc partials of basis k, scale by norm C_k and map to the reference's
// parameter order: vech(dF/dL_k) = vech(2 G L_k) + diag(1.5 D / L_ii), then
// dF/ds_k (python/make_grad.py:61-79 output layout, GRADA block k).
template <int N>
__global__ void __launch_bounds__(128) grad_reduce_kernel(const double *__restrict__ part,
                                                          int nlc, int K,
                                                          const double *__restrict__ bra,
                                                          const double *__restrict__ C,
                                                          const double *__restrict__ scal,
                                                          double scale_override,
                                                          double *__restrict__ g, int *status) {
    using BL = BraLayout<N>;
    constexpr int PS = tri(N) + 1 + 3 * N;
    constexpr int blk = tri(N) + 3 * N;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    double acc[PS];
#pragma unroll
    for (int t = 0; t < PS; ++t) acc[t] = 0.0;
    for (int lc = 0; lc < nlc; ++lc) {
        const double *p = part + (size_t)lc * PS * K + k;
#pragma unroll
        for (int t = 0; t < PS; ++t) acc[t] += p[(size_t)t * K];
    }
    const double norm = scale_override != 0.0 ? scale_override : scal[1];
    const double sc = norm * (C ? C[k] : 1.0);
    double L[tri(N)];
#pragma unroll
    for (int t = 0; t < tri(N); ++t) L[t] = bra[(BL::L + t) * (size_t)K + k];
    double *o = g + (size_t)k * blk;
    int idx = 0;
    bool fin = true;
#pragma unroll
    for (int j = 0; j < N; ++j)
#pragma unroll
        for (int i = j; i < N; ++i) {
            // (2 G L)_ij with G symmetric packed in acc[0..tri)
            double s = 0.0;
#pragma unroll
            for (int a = 0; a <= j; ++a) s += acc[sx(i, a)] * L[sx(j, a)];
            s *= 2.0;
            if (i == j) s += 1.5 * acc[tri(N)] / L[sx(i, i)];
            const double v = sc * s;
            fin = fin && isfinite(v);
            o[idx++] = v;
        }
#pragma unroll
    for (int t = 0; t < 3 * N; ++t) {
        const double v = sc * acc[tri(N) + 1 + t];
        fin = fin && isfinite(v);
        o[tri(N) + t] = v;
    }
    if (!fin) atomicOr(status, 2);
}

// ---------------------------------------------------------------------------
// Per-term elements for the matel / gradel API: terms[3 t .. 3 t + 2] =
// (stf, ii, jj), 1-based as in python/matel.py:28 and python/gradel.py:27.
template <int N>
__global__ void __launch_bounds__(128) matel_kernel(const int *__restrict__ terms, int nterms,
                                                    int K, int nst, Consts<N> cs,
                                                    const double *__restrict__ bra,
                                                    const double *__restrict__ ket,
                                                    double *__restrict__ out, int *status) {
    using KL = KetLayout<N>;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nterms) return;
    const int stf = terms[3 * t] - 1, ii = terms[3 * t + 1] - 1, jj = terms[3 * t + 2] - 1;
    if (stf < 0 || stf >= nst || ii < 0 || ii >= K || jj < 0 || jj >= K) {
        atomicOr(status, 4);
        for (int q = 0; q < 4; ++q) out[4 * t + q] = NAN;
        return;
    }
    const BraRef b{bra + ii, (size_t)K};
    const double *kr = ket + ((size_t)jj * nst + stf) * KL::size;
    double ov, tau, rho, sig;
    if (!term_energy<N>(b, kr, cs, ov, tau, rho, sig)) flag_bad_pair(status, 1, ii * K + jj);
    out[4 * t + 0] = ov;
    out[4 * t + 1] = 2.0 * ov * tau;
    out[4 * t + 2] = ov * rho;
    out[4 * t + 3] = ov * sig;
}

template <int N>
__global__ void __launch_bounds__(128) gradel_kernel(const int *__restrict__ terms, int nterms,
                                                     int K, int nst, Consts<N> cs,
                                                     const double *__restrict__ bra,
                                                     const double *__restrict__ ket,
                                                     double *__restrict__ tgvl,
                                                     double *__restrict__ tgvls, int *status) {
    using KL = KetLayout<N>;
    using BL = BraLayout<N>;
    constexpr int blk = tri(N) + 3 * N;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nterms) return;
    const int stf = terms[3 * t] - 1, ii = terms[3 * t + 1] - 1, jj = terms[3 * t + 2] - 1;
    if (stf < 0 || stf >= nst || ii < 0 || ii >= K || jj < 0 || jj >= K) {
        atomicOr(status, 4);
        for (int q = 0; q < blk; ++q) tgvl[(size_t)t * blk + q] = tgvls[(size_t)t * blk + q] = NAN;
        return;
    }
    const BraRef b{bra + ii, (size_t)K};
    const double *kr = ket + ((size_t)jj * nst + stf) * KL::size;
    double L[tri(N)];
#pragma unroll
    for (int q = 0; q < tri(N); ++q) L[q] = bra[(BL::L + q) * (size_t)K + ii];
    const double dbl = (ii == jj) ? 2.0 : 1.0;  // python/gradel.py:388-390
#pragma unroll
    for (int which = 0; which < 2; ++which) {
        double accG[tri(N)], accS[3 * N], accD = 0.0;
#pragma unroll
        for (int q = 0; q < tri(N); ++q) accG[q] = 0.0;
#pragma unroll
        for (int q = 0; q < 3 * N; ++q) accS[q] = 0.0;
        // which 0: dH (lam 1, E 0); which 1: dS (lam 0, E -1)
        if (!term_grad<N>(b, kr, cs, which == 0 ? 1.0 : 0.0, which == 0 ? 0.0 : -1.0, 1.0, accG,
                          accD, accS))
            flag_bad_pair(status, 1, ii * K + jj);
        double *o = (which == 0 ? tgvl : tgvls) + (size_t)t * blk;
        int idx = 0;
#pragma unroll
        for (int j = 0; j < N; ++j)
#pragma unroll
            for (int i = j; i < N; ++i) {
                double s = 0.0;
#pragma unroll
                for (int a = 0; a <= j; ++a) s += accG[sx(i, a)] * L[sx(j, a)];
                s *= 2.0;
                if (i == j) s += 1.5 * accD / L[sx(i, i)];
                o[idx++] = dbl * s;
            }
#pragma unroll
        for (int q = 0; q < 3 * N; ++q) o[tri(N) + q] = dbl * accS[q];
    }
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
void launch_fp64_probe(int blocks, int iters, double *sink, cudaStream_t st) {
    fp64_probe_kernel<<<blocks, 256, 0, st>>>(iters, 1.0, sink);
}

// Boys function on an array (python/utils.py:78-106)
__global__ void f0_kernel(const double *__restrict__ z, int count, double *__restrict__ f,
                          double *__restrict__ df) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const double zz = z[i];
    // evaluate with a = 1 so that fs = F0(z), dfs = F0'(z)
    double fs, dfs, ia, zo;
    boys<true>(1.0, zz, fs, dfs, ia, zo);
    if (f) f[i] = fs;
    if (df) df[i] = dfs;
}

// ---------------------------------------------------------------------------
// Host-side launchers (one instantiation per supported particle count)
template <int N>
Consts<N> make_consts(const double *mass, const double *ncv, double efs) {
    Consts<N> c;
    for (int i = 0; i < N * N; ++i) c.M[i] = mass[i];
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
        prep_ket_kernel<N><<<(nk + 127) / 128, 128, 0, st>>>(a.iv, a.C, a.K, a.nst, cs, a.sml,
                                                             a.sms, a.scvv, a.ket);
    }
    static void energy(const LaunchArgs &a, cudaStream_t st) {
        Consts<N> cs = make_consts<N>(a.mass_h, a.ncv_h, a.efs);
        const int threads = 128, wpb = threads / 32;
        energy_kernel<N><<<(a.ntiles + wpb - 1) / wpb, threads, 0, st>>>(
            a.tiles, a.ntiles, a.LC_e, a.K, a.nst, cs, a.bra, a.ket, a.H, a.S, a.Kin, a.Pot,
            a.status);
    }
    static void grad_tiles(const LaunchArgs &a, cudaStream_t st) {
        Consts<N> cs = make_consts<N>(a.mass_h, a.ncv_h, a.efs);
        const int nkb = (a.K + 31) / 32, nlc = (a.K + a.LC_g - 1) / a.LC_g;
        const int threads = 128, wpb = threads / 32;
        grad_kernel<N><<<(nkb * nlc + wpb - 1) / wpb, threads, 0, st>>>(
            nkb, nlc, a.LC_g, a.K, a.nst, cs, a.bra, a.ket, a.scal, a.lam, a.part, a.status);
    }
    static void grad_reduce(const LaunchArgs &a, cudaStream_t st) {
        const int nlc = (a.K + a.LC_g - 1) / a.LC_g;
        grad_reduce_kernel<N><<<(a.K + 127) / 128, 128, 0, st>>>(
            a.part, nlc, a.K, a.bra, a.C, a.scal, a.scale_override, a.g, a.status);
    }
    static void grad(const LaunchArgs &a, cudaStream_t st) {
        grad_tiles(a, st);
        grad_reduce(a, st);
    }
    static void matel(const LaunchArgs &a, const int *terms, int nterms, double *out,
                      cudaStream_t st) {
        Consts<N> cs = make_consts<N>(a.mass_h, a.ncv_h, a.efs);
        matel_kernel<N><<<(nterms + 127) / 128, 128, 0, st>>>(terms, nterms, a.K, a.nst, cs,
                                                              a.bra, a.ket, out, a.status);
    }
    static void gradel(const LaunchArgs &a, const int *terms, int nterms, double *tg,
                       double *tgs, cudaStream_t st) {
        Consts<N> cs = make_consts<N>(a.mass_h, a.ncv_h, a.efs);
        gradel_kernel<N><<<(nterms + 127) / 128, 128, 0, st>>>(terms, nterms, a.K, a.nst, cs,
                                                               a.bra, a.ket, tg, tgs, a.status);
    }
};

#define NECG_DISPATCH(n, call)                  \
    switch (n) {                                \
    case 1: Launch<1>::call; break;             \
    case 2: Launch<2>::call; break;             \
    case 3: Launch<3>::call; break;             \
    case 4: Launch<4>::call; break;             \
    case 5: Launch<5>::call; break;             \
    case 6: Launch<6>::call; break;             \
    default: return -1;                         \
    }

int launch_prep(const LaunchArgs &a, cudaStream_t st) {
    NECG_DISPATCH(a.n, prep(a, st));
    return 0;
}
int launch_energy(const LaunchArgs &a, cudaStream_t st) {
    NECG_DISPATCH(a.n, energy(a, st));
    return 0;
}
int launch_grad(const LaunchArgs &a, cudaStream_t st) {
    NECG_DISPATCH(a.n, grad(a, st));
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
int launch_matel(const LaunchArgs &a, const int *terms, int nterms, double *out,
                 cudaStream_t st) {
    NECG_DISPATCH(a.n, matel(a, terms, nterms, out, st));
    return 0;
}
int launch_gradel(const LaunchArgs &a, const int *terms, int nterms, double *tg, double *tgs,
                  cudaStream_t st) {
    NECG_DISPATCH(a.n, gradel(a, terms, nterms, tg, tgs, st));
    return 0;
}
void launch_rows_finalize(const LaunchArgs &a, double *f_out, double *gradc, int given,
                          double eng, double norm, cudaStream_t st) {
    rows_kernel<<<(a.K * 32 + 255) / 256, 256, 0, st>>>(a.H, a.S, a.C, a.K, a.rows);
    finalize_kernel<<<1, 1024, 0, st>>>(a.rows, a.C, a.K, a.scal, f_out, gradc, a.status, given,
                                        eng, norm);
}

__global__ void reset_status_kernel(int *status) {
    status[0] = 0;
    status[1] = 0x7fffffff;
}
void launch_reset_status(int *status, cudaStream_t st) { reset_status_kernel<<<1, 1, 0, st>>>(status); }
void launch_f0(const double *z, int count, double *f, double *df, cudaStream_t st) {
    f0_kernel<<<(count + 255) / 256, 256, 0, st>>>(z, count, f, df);
}

}  // namespace necg

namespace necg {
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
