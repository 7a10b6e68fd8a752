// necg_math.cuh -- per-term FP64 math of the ECG energy+gradient path.
//
// One "term" is a (bra k, ket l, symmetry P) triple: the reference's
// matel(stf, k, l) (python/matel.py:28-210) and the bra part of
// gradel(stf, k, l) (python/gradel.py:27-392).  The reference expands every
// n x n matrix to 3n x 3n with kron(., I3) and inverts with LAPACK; here all
// work stays in n-space with the shifts viewed as n x 3 matrices, B = A_k + A_l'
// is factored by Cholesky in registers, and the gradient is formed with respect
// to A_k = L_k L_k^T (a symmetric n x n matrix) and s_k, then mapped to vech(L_k)
// once per basis function (dF/dL = 2 G L).
//
// Notation (n = N particles):
//   A_k, A_l' = P^T A_l P    symmetric, packed lower (N(N+1)/2)
//   S_k, S_l' = sms s_l      n x 3 (row = particle, column = x, y, z)
//   B = A_k + A_l', Bi = B^-1, T = Bi (A_k S_k + A_l' S_l')   (st in the reference)
//   Dk = S_k - T, Dl = T - S_l', Y = A_l' Dl (= A_k Dk)
//   ov  = sqrt(8^n) (|L_k| |L_l|)^{3/2} / |B|^{3/2} exp(<E,T> - i1 - i2)
//   tau = 3 tr(M X) - 2 <Y, M Y>, X = A_k Bi A_l',   tk = 2 ov tau
//   rho = sum_v c_v F0(|v^T T|^2 / v^T Bi v) (v^T Bi v)^{-1/2}, ert = ov rho
//   sig = efs sum_i q_i T[i,z],  zht = ov sig
// Coulomb pairs v: e_q (nucleus-particle) or e_p - e_q (particle-particle),
// c_v = 2 q_p q_q / sqrt(pi).
//
// Bra gradient of F = w (h - E ov) with h = tk + ert - zht:
//   dF/dA_k = Fw (-Dk Dk^T - 1.5 Bi + 0.75 A_k^-1)
//             + ovw (Bi (6 N_l' + W) Bi + Qk Dk^T + Dk Qk^T)
//   dF/ds_k = -2 Fw Y + 2 ovw A_k Qk
//   N_l' = A_l' M A_l',  Qk = Bi (Z' - 4 A_l' M Y),
//   Z' = sum_v alpha_v v b_v^T - (efs/2) q e_z^T,  W = sum_v beta_v v v^T,
//   alpha_v = c_v F0'(z) a^{-3/2},  beta_v = c_v a^{-3/2} (z F0'(z) + F0(z)/2).
// The A_k^-1 term (coefficient D = 0.75 Fw) maps to vech(dF/dL) as 2 D / L_ii
// on the diagonal only, so it is kept as one scalar per basis function.
//
// All term functions are templates over the scalar type R and over the bra and
// ket accessors.  The kernels instantiate them with R = double; the operation
// counter in the C-ABI layer instantiates them with a counting scalar on the
// host, so the algorithmic FLOP count is taken from this very code.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#ifdef __CUDACC__
#define NECG_HD __host__ __device__ __forceinline__
#else
#define NECG_HD inline
#endif

namespace necg {

__host__ __device__ constexpr int tri(int n) { return n * (n + 1) / 2; }
// packed lower-triangular, row-major: (i, j) with i >= j
__host__ __device__ constexpr int sx(int i, int j) {
    return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i;
}

// Pade coefficients of the Boys function F0 (python/shared.py:76-86,
// source/error_function_approximation.f90) and its branch point
// (python/utils.py:85).
#define NECG_PC1 0.564691197e-04
#define NECG_PC2 0.758433197e-03
#define NECG_PC3 0.769838037e-02
#define NECG_PC4 0.629344460e-01
#define NECG_PC5 0.213271302e+00
#define NECG_PC6 0.720266520e-04
#define NECG_PC7 0.955528842e-03
#define NECG_PC8 0.101431553e-01
#define NECG_PC9 0.738522953e-01
#define NECG_PC10 0.338450368e+00
#define NECG_PC11 0.879937801e+00
#define NECG_F0_SPLIT 16.3578
#define NECG_PI 3.141592653589793
#define NECG_SQRT_PI 1.7724538509055159

// Ket record: one per (l, P), read warp-uniformly by the tile kernels.
// Layout (doubles): Ap[tri] Sp[3N] ASp[3N] Np[tri] AMn4[N*N] i2 pre tMA w wC winv pad
// (AMn4 = -4 A_l' M, row-major: the factor of Z's update folded in, so that the
// update is one FMA chain per output)
template <int N> struct KetLayout {
    static constexpr int T = tri(N);
    static constexpr int Ap = 0;
    static constexpr int Sp = Ap + T;
    static constexpr int ASp = Sp + 3 * N;
    static constexpr int Np = ASp + 3 * N;
    static constexpr int AMn4 = Np + T;
    static constexpr int i2 = AMn4 + N * N;
    static constexpr int pre = i2 + 1;
    static constexpr int tMA = pre + 1;  // tr(M A_l')
    static constexpr int w = tMA + 1;    // symmetry weight scvv[P]
    static constexpr int wC = w + 1;     // 2 scvv[P] C_l (gradient weight)
    static constexpr int winv = wC + 1;  // scvv[P^-1] (ket weight of the symmetric pass)
    static constexpr int size = (winv + 1 + 1) & ~1;  // even, 16-byte records
};

// Bra record: structure of arrays over k, field f of basis k at f*K + k.
template <int N> struct BraLayout {
    static constexpr int T = tri(N);
    static constexpr int A = 0;
    static constexpr int S = A + T;
    static constexpr int AS = S + 3 * N;
    static constexpr int Nk = AS + 3 * N;  // A_k M A_k
    static constexpr int i1 = Nk + T;
    static constexpr int pre = i1 + 1;
    static constexpr int tMA = pre + 1;
    static constexpr int L = tMA + 1;      // L_k, packed lower
    static constexpr int size = L + T;
};

// Per-problem constants, passed to kernels by value (constant bank).
template <int N> struct Consts {
    double M[N * N];    // inverse-mass tensor, row-major
    double M4[N * N];   // 4 M (Q_l = Q_k + 4 M Y as one FMA chain per output)
    double Mq[tri(N)];  // packed lower: M_ii on the diagonal, M_ik + M_ki below (quadratic forms in M)
    double cv[tri(N)];  // c_v for the n(n+1)/2 Coulomb pairs (p<q, q-major order)
    double q[N];        // ncv[1..n]
    double efs;
    double sqrt8n;      // sqrt(8^n)
    // M4 and Mq from M
    NECG_HD void derive() {
        for (int i = 0; i < N * N; ++i) M4[i] = 4.0 * M[i];
        for (int i = 0; i < N; ++i)
            for (int k = 0; k <= i; ++k) Mq[sx(i, k)] = i == k ? M[i * N + i] : M[i * N + k] + M[k * N + i];
    }
};

// Doubles of one part's compact output for one tile of a split lockstep group
// of the fused pass (ps = tri(n) + 1 + 3n fields, lc kets per tile): ket
// partials, then H and S sums.
__host__ __device__ inline size_t fsym_tail_slot(int ps, int lc) {
    return (size_t)lc * 2 * ps + (size_t)lc * 64;
}

// Coulomb pair enumeration order: for q = 1..N, p = 0..q-1  -> index q(q-1)/2 + p
__host__ __device__ constexpr int vidx(int p, int q) { return q * (q - 1) / 2 + p; }

// ---------------------------------------------------------------------------
// Device accessors
#ifdef __CUDACC__
// Bra fields are per-lane and invariant over a tile's ket loops; holding them in
// registers would cost 2 (6N + 2 tri(N)) registers, so they are re-read from the
// (L1-resident) structure-of-arrays at the point of use.  The volatile asm keeps
// the compiler from hoisting the loads out of the ket loops.
__device__ __forceinline__ double ldv(const double *p) {
    double v;
    asm volatile("ld.global.nc.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
struct BraRef {
    const double *p;  // bra + k
    size_t K;
    __device__ __forceinline__ double operator()(int f) const { return ldv(p + (size_t)f * K); }
};
// Bra record staged in shared memory (field f of this lane at p[f * 32]), read
// at the point of use through a volatile shared load (not hoisted into registers).
struct BraSmem {
    const double *p;  // shared base + lane
    __device__ __forceinline__ double operator()(int f) const {
        double v;
        const unsigned a = (unsigned)__cvta_generic_to_shared(p + f * 32);
        asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a));
        return v;
    }
};
// Ket record staged in shared memory by its warp, read at the point of use
// (a broadcast shared load, not hoisted into registers).
struct KetSmem {
    const double *p;
    __device__ __forceinline__ double operator[](int i) const {
        double v;
        const unsigned a = (unsigned)__cvta_generic_to_shared(p + i);
        asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a));
        return v;
    }
};
// Ket record read at the point of use (warp-uniform, L1 broadcast), so its
// fields do not stay live in registers between their uses within a term.
struct KetRefV {
    const double *p;
    __device__ __forceinline__ double operator[](int i) const { return ldv(p + i); }
};
#endif

// Register accumulators of one bra gradient (see term_grad).
template <int N, typename R> struct RegAcc {
    R G[tri(N)], D, S[3 * N];
#pragma nv_exec_check_disable
    NECG_HD void zero() {
#pragma unroll
        for (int t = 0; t < tri(N); ++t) G[t] = R(0.0);
        D = R(0.0);
#pragma unroll
        for (int t = 0; t < 3 * N; ++t) S[t] = R(0.0);
    }
    NECG_HD R &g(int t) { return G[t]; }
    NECG_HD R &d() { return D; }
    NECG_HD R &s(int t) { return S[t]; }
};

// ---------------------------------------------------------------------------
// x^(-1/2) for normal, positive x.  On the device the hardware approximation
// rsqrt.approx.ftz.f64 (relative error below 1e-6) is refined by one step of
// Householder's third-order iteration for 1/sqrt(x): with r = 1 - x y^2,
// y <- y + y r (1/2 + 3/8 r), the series of (1 - r)^(-1/2) to second order,
// whose truncation error (of order r^3) lies far below the result's rounding.
// Measured on a B200 over 2^24 inputs in [2^-40, 2^40]: within 2 ulp of
// rsqrt(double) and 2.4 ulp of 1 / sqrt(x), at 1.56x its throughput.  Host
// builds (the emulator) use 1 / sqrt(x).
NECG_HD double rsq(double x) {
#ifdef __CUDA_ARCH__
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double r = fma(-(x * y), y, 1.0);
    return fma(y * r, fma(0.375, r, 0.5), y);
#else
    return 1.0 / ::sqrt(x);
#endif
}

// 1/x for normal, positive x.  On the device the hardware approximation
// rcp.approx.ftz.f64 is refined by one third-order step: with e = 1 - x y,
// y <- y + y (e + e^2), the series of 1 / (1 - e) to second order, whose
// truncation error (of order e^3) lies far below the result's rounding.  Host
// builds (the emulator) use 1 / x.
NECG_HD double rcp(double x) {
#ifdef __CUDA_ARCH__
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x, y, 1.0);
    return fma(y, fma(e, e, e), y);
#else
    return 1.0 / x;
#endif
}

// Cholesky of a packed SPD matrix B = R R^T; returns the inverse Bi (packed),
// prod(1/R_ii) and a success flag.  Fully unrolled into registers.
#pragma nv_exec_check_disable
template <int N, typename R>
NECG_HD bool chol_inverse(const R (&B)[tri(N)], R (&Bi)[tri(N)], R &prod_rinv) {
    R Rm[tri(N)];
    R rinv[N];
    bool ok = true;
#pragma unroll
    for (int j = 0; j < N; ++j) {
        R d = B[sx(j, j)];
#pragma unroll
        for (int k = 0; k < j; ++k) d -= Rm[sx(j, k)] * Rm[sx(j, k)];
        const bool pos = d > 0.0;
        ok = ok && pos;
        if (!pos) d = R(1.0);
        const R r = rsq(d);
        rinv[j] = r;
        Rm[sx(j, j)] = d * r;
#pragma unroll
        for (int i = j + 1; i < N; ++i) {
            R s = B[sx(i, j)];
#pragma unroll
            for (int k = 0; k < j; ++k) s -= Rm[sx(i, k)] * Rm[sx(j, k)];
            Rm[sx(i, j)] = s * r;
        }
    }
    // W = R^-1 (lower triangular), in place
#pragma unroll
    for (int j = 0; j < N; ++j) {
        Rm[sx(j, j)] = rinv[j];
#pragma unroll
        for (int i = j + 1; i < N; ++i) {
            R s = Rm[sx(i, j)] * rinv[j];
#pragma unroll
            for (int k = j + 1; k < i; ++k) s += Rm[sx(i, k)] * Rm[sx(k, j)];
            Rm[sx(i, j)] = -(s * rinv[i]);
        }
    }
    // Bi = W^T W : Bi_ij = sum_{k >= max(i,j)} W_ki W_kj
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            R s = Rm[sx(i, i)] * Rm[sx(i, j)];
#pragma unroll
            for (int k = i + 1; k < N; ++k) s += Rm[sx(k, i)] * Rm[sx(k, j)];
            Bi[sx(i, j)] = s;
        }
    R p = rinv[0];
#pragma unroll
    for (int j = 1; j < N; ++j) p *= rinv[j];
    prod_rinv = p;
    return ok;
}

// y = S x for S symmetric (packed, read through an accessor) and x n x 3
#pragma nv_exec_check_disable
template <int N, typename R, typename Acc>
NECG_HD void symv3(const Acc &S, int off, const R (&x)[3 * N], R (&y)[3 * N]) {
    // each element of S is read once and used for the three columns (the
    // accessors may load from memory at every call)
#pragma unroll
    for (int i = 0; i < N; ++i) {
        {
            const R a = S[off + sx(i, 0)];
#pragma unroll
            for (int c = 0; c < 3; ++c) y[3 * i + c] = a * x[c];
        }
#pragma unroll
        for (int k = 1; k < N; ++k) {
            const R a = S[off + sx(i, k)];
#pragma unroll
            for (int c = 0; c < 3; ++c) y[3 * i + c] += a * x[3 * k + c];
        }
    }
}

// y += S x for S symmetric (packed, read through an accessor) and x n x 3: the
// products fuse into y's values
#pragma nv_exec_check_disable
template <int N, typename R, typename Acc>
NECG_HD void symv3_acc(const Acc &S, int off, const R (&x)[3 * N], R (&y)[3 * N]) {
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const R a = S[off + sx(i, k)];
#pragma unroll
            for (int c = 0; c < 3; ++c) y[3 * i + c] += a * x[3 * k + c];
        }
}

// Boys-function pieces for one Coulomb pair.  Given a = v^T Bi v and
// bb = |v^T T|^2 (z = bb / a) returns fs = F0(z) a^{-1/2} and, when GRAD,
// D = F0'(z) / F0(z) (so F0'(z) a^{-1/2} = fs D) and ia = 1/a.  The Pade branch
// (z <= 16.3578) and the asymptotic branch sqrt(pi/(4z)) follow
// python/utils.py:78-106; in the Pade branch F0 = sqrt(num / den), and from
// F0^2 = num / den, F0' = F0 (num'/num - den'/den) / 2, so
//   D = F0' / F0 = (num' den - den' num) / (2 num den)  (Pade),  -1 / (2 z)  (asymptotic),
// with num'/2 den - den'/2 num evaluated as one polynomial.  Two
// special functions give every quotient and root; RCP chooses between two ways:
//   RCP:   ia = 1/a (rcp);  q = (num den a)^{-1/2} (Pade) or bb^{-1/2}:
//          fs = num q or (sqrt(pi) / 2) q, and q^2 a = 1 / (num den) or 1 / z;
//   !RCP:  ra = a^{-1/2}, ia = ra^2;  q = (num den)^{-1/2} or bb^{-1/2}:
//          fs = num q ra or (sqrt(pi) / 2) q, and q^2 = 1 / (num den) or 1 / bb.
// RCP takes four FP64 operations fewer per pair but holds more values at once;
// it is used where it timed faster on a B200 (n > 3).  The branch is taken per
// lane: every lane evaluates the Pade polynomials and the two forms differ only
// in the operand of the square root and in the factors selected, so that the
// lanes of a warp on either side of the split run the same instructions.
template <typename R> NECG_HD void boys_pade(R z, R &num, R &den) {
    num = ((((NECG_PC1 * z + NECG_PC2) * z + NECG_PC3) * z + NECG_PC4) * z + NECG_PC5) * z + 1.0;
    den = (((((NECG_PC6 * z + NECG_PC7) * z + NECG_PC8) * z + NECG_PC9) * z + NECG_PC10) * z + NECG_PC11) * z + 1.0;
}
// (num' den - den' num) / 2 as one polynomial of degree 10: its coefficients
// are those of num'/2 den - den'/2 num, formed from the Pade coefficients when
// the code is compiled
struct BoysDP {
    double c[11];
    constexpr BoysDP() : c{} {
        const double nh[5] = {0.5 * NECG_PC5, NECG_PC4, 1.5 * NECG_PC3, 2.0 * NECG_PC2, 2.5 * NECG_PC1};  // num'/2
        const double de[7] = {1.0, NECG_PC11, NECG_PC10, NECG_PC9, NECG_PC8, NECG_PC7, NECG_PC6};       // den
        const double dh[6] = {0.5 * NECG_PC11, NECG_PC10, 1.5 * NECG_PC9, 2.0 * NECG_PC8, 2.5 * NECG_PC7,
                              3.0 * NECG_PC6};                                                         // den'/2
        const double nu[6] = {1.0, NECG_PC5, NECG_PC4, NECG_PC3, NECG_PC2, NECG_PC1};                  // num
        for (int i = 0; i < 5; ++i)
            for (int j = 0; j < 7; ++j) c[i + j] += nh[i] * de[j];
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) c[i + j] -= dh[i] * nu[j];
    }
};
template <typename R> NECG_HD R boys_pade_dp(R z) {
    constexpr BoysDP p{};
    R v = R(p.c[10]) * z + p.c[9];
#pragma unroll
    for (int k = 8; k >= 0; --k) v = v * z + p.c[k];
    return v;
}
#pragma nv_exec_check_disable
template <bool GRAD, bool RCP = true, typename R>
NECG_HD void boys(R a, R bb, R &fs, R &D, R &ia, R &z) {
    R ra = R(1.0);
    if constexpr (RCP) {
        ia = rcp(a);
    } else {
        ra = rsq(a);
        ia = ra * ra;
    }
    z = bb * ia;
    const bool pade = z <= NECG_F0_SPLIT;
    R num, den;
    boys_pade(z, num, den);
    const R c = R(0.5 * NECG_SQRT_PI);
    R q;
    if constexpr (RCP) {
        q = rsq(pade ? (num * den) * a : bb);
        fs = (pade ? num : c) * q;
    } else {
        q = rsq(pade ? num * den : bb);
        const R fp = (num * q) * ra, fa = c * q;
        fs = pade ? fp : fa;
    }
    if (GRAD) {
        const R P = boys_pade_dp(z);
        R dp, da;
        if constexpr (RCP) {
            const R qa = (q * q) * a;
            dp = qa * P;
            da = -0.5 * qa;
        } else {
            const R qq = q * q;
            dp = qq * P;
            da = -0.5 * a * qq;
        }
        D = pade ? dp : da;
    } else {
        D = R(0.0);
    }
}

// Coulomb sum with the pieces of its derivative (python/gradel.py:266-337):
// rho = sum_v c_v F0(z_v) a_v^-1/2, Z' = sum_v alpha_v v b_v^T - (efs/2) q e_z^T
// (the Stark part folded in), W = sum_v beta_v v v^T (packed).
#pragma nv_exec_check_disable
template <int N, typename R>
NECG_HD void coulomb_grad(const R (&Bi)[tri(N)], const R (&T)[3 * N], const Consts<N> &cs, R &rho,
                          R (&Z)[3 * N], R (&W)[tri(N)]) {
#pragma unroll
    for (int t = 0; t < 3 * N; ++t) Z[t] = R(0.0);
#pragma unroll
    for (int t = 0; t < tri(N); ++t) W[t] = R(0.0);
    rho = R(0.0);
#pragma unroll
    for (int q = 1; q <= N; ++q)
#pragma unroll
        for (int p = 0; p < q; ++p) {
            R a = Bi[sx(q - 1, q - 1)];
            R bv[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) bv[c] = T[3 * (q - 1) + c];
            if (p > 0) {
                a += Bi[sx(p - 1, p - 1)] - 2.0 * Bi[sx(q - 1, p - 1)];
#pragma unroll
                for (int c = 0; c < 3; ++c) bv[c] -= T[3 * (p - 1) + c];
            }
            const R bb = bv[0] * bv[0] + bv[1] * bv[1] + bv[2] * bv[2];
            R fs, D, ia, z;
            boys<true, (N > 3)>(a, bb, fs, D, ia, z);
            // alpha = c F0' a^{-3/2} = c fs D / a, beta = c a^{-3/2} (z F0' + F0 / 2) = (c fs / a)(z D + 1/2)
            const R cf = cs.cv[vidx(p, q)] * fs;
            rho += cf;
            const R cfi = cf * ia;
            const R al = cfi * D;
            const R be = cfi * (D * z + 0.5);
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) Z[3 * (q - 1) + cc] += al * bv[cc];
            W[sx(q - 1, q - 1)] += be;
            if (p > 0) {
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) Z[3 * (p - 1) + cc] -= al * bv[cc];
                W[sx(p - 1, p - 1)] += be;
                W[sx(q - 1, p - 1)] -= be;
            }
        }
#pragma unroll
    for (int i = 0; i < N; ++i) Z[3 * i + 2] -= 0.5 * cs.efs * cs.q[i];
}

// acc += Bi Mt Bi (Mt packed symmetric), column by column of Mt Bi.
#pragma nv_exec_check_disable
template <int N, typename R, typename OUT>
NECG_HD void sandwich(const R (&Bi)[tri(N)], const R (&Mt)[tri(N)], OUT &&add) {
#pragma unroll
    for (int j = 0; j < N; ++j) {
        R col[N];
#pragma unroll
        for (int a = 0; a < N; ++a) {
            R s = Mt[sx(a, 0)] * Bi[sx(0, j)];
#pragma unroll
            for (int k = 1; k < N; ++k) s += Mt[sx(a, k)] * Bi[sx(k, j)];
            col[a] = s;
        }
#pragma unroll
        for (int i = j; i < N; ++i) {
            R s = Bi[sx(i, 0)] * col[0];
#pragma unroll
            for (int a = 1; a < N; ++a) s += Bi[sx(i, a)] * col[a];
            add(sx(i, j), s);
        }
    }
}

// The same with each output's sum started from seed(t) (an accumulator's value,
// so the products fuse into it): put(t, seed(t) + (Bi Mt Bi)_t).
#pragma nv_exec_check_disable
template <int N, typename R, typename SEED, typename OUT>
NECG_HD void sandwich_seeded(const R (&Bi)[tri(N)], const R (&Mt)[tri(N)], SEED &&seed, OUT &&put) {
#pragma unroll
    for (int j = 0; j < N; ++j) {
        R col[N];
#pragma unroll
        for (int a = 0; a < N; ++a) {
            R s = Mt[sx(a, 0)] * Bi[sx(0, j)];
#pragma unroll
            for (int k = 1; k < N; ++k) s += Mt[sx(a, k)] * Bi[sx(k, j)];
            col[a] = s;
        }
#pragma unroll
        for (int i = j; i < N; ++i) {
            R s = seed(sx(i, j));
#pragma unroll
            for (int a = 0; a < N; ++a) s += Bi[sx(i, a)] * col[a];
            put(sx(i, j), s);
        }
    }
}

// B = A_k + A_l', its inverse, T = Bi (A_k S_k + A_l' S_l') and the overlap.
#pragma nv_exec_check_disable
template <int N, typename R, typename BA, typename KA>
NECG_HD bool term_core(const BA &b, const KA &kr, const Consts<N> &cs, R (&Bi)[tri(N)],
                       R (&T)[3 * N], R &ov) {
    using KL = KetLayout<N>;
    using BL = BraLayout<N>;
    R prinv;
    bool ok;
    {
        R B[tri(N)];
#pragma unroll
        for (int t = 0; t < tri(N); ++t) B[t] = b(BL::A + t) + kr[KL::Ap + t];
        ok = chol_inverse<N>(B, Bi, prinv);
    }
    R Ev[3 * N];
#pragma unroll
    for (int t = 0; t < 3 * N; ++t) Ev[t] = b(BL::AS + t) + kr[KL::ASp + t];
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            R s = Bi[sx(i, 0)] * Ev[c];
#pragma unroll
            for (int k = 1; k < N; ++k) s += Bi[sx(i, k)] * Ev[3 * k + c];
            T[3 * i + c] = s;
        }
    R i3 = Ev[0] * T[0];
#pragma unroll
    for (int t = 1; t < 3 * N; ++t) i3 += Ev[t] * T[t];
    const R p3 = prinv * prinv * prinv;
    ov = cs.sqrt8n * b(BL::pre) * kr[KL::pre] * p3 * exp(i3 - b(BL::i1) - kr[KL::i2]);
    return ok;
}

// tau = 3 tr(M X) - 2 <Y, M Y>.  tr(M X) with X = A_k Bi A_l' is written through
// the matrix with the smaller tr(M A): X = A_s - A_s Bi A_s, which keeps the
// subtraction free of cancellation.  The choice differs from lane to lane, so
// both N_s are read and one is selected (no divergent branch).  Y = A_l' (T - S_l')
// is returned for the gradient formulas.
#pragma nv_exec_check_disable
template <int N, typename R, typename BA, typename KA>
NECG_HD R term_tau(const BA &b, const KA &kr, const Consts<N> &cs, const R (&Bi)[tri(N)],
                   const R (&T)[3 * N], R (&Y)[3 * N]) {
    using KL = KetLayout<N>;
    using BL = BraLayout<N>;
    R tMX;
    {
        const R tl = kr[KL::tMA], tk = b(BL::tMA);
        const bool use_l = tl <= tk;
        // tr(Bi N_s): the diagonal and the off-diagonal products summed apart
        R dg = R(0.0), od = R(0.0);
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
            for (int j = 0; j <= i; ++j) {
                const R nl = kr[KL::Np + sx(i, j)], nk = b(BL::Nk + sx(i, j));
                const R v = Bi[sx(i, j)] * (use_l ? nl : nk);
                if (i == j)
                    dg = (i == 0) ? v : dg + v;
                else
                    od = (i == 1) ? v : od + v;
            }
        tMX = (use_l ? tl : tk) - (dg + 2.0 * od);
    }
    R yMy = R(0.0);
    {
        // Y = A_l' (T - S_l') = A_l' T - A_l' S_l', the second product from the ket record
#pragma unroll
        for (int t = 0; t < 3 * N; ++t) Y[t] = -kr[KL::ASp + t];
        symv3_acc<N>(kr, KL::Ap, T, Y);
        // <Y, M Y> = sum_c sum_i Y_ic (M_ii Y_ic + sum_{k<i} (M_ik + M_ki) Y_kc)
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                R s = cs.Mq[sx(i, i)] * Y[3 * i + c];
#pragma unroll
                for (int k = 0; k < i; ++k) s += cs.Mq[sx(i, k)] * Y[3 * k + c];
                yMy += Y[3 * i + c] * s;
            }
    }
    return 3.0 * tMX - 2.0 * yMy;
}
#pragma nv_exec_check_disable
template <int N, typename R, typename BA, typename KA>
NECG_HD R term_tau(const BA &b, const KA &kr, const Consts<N> &cs, const R (&Bi)[tri(N)],
                   const R (&T)[3 * N]) {
    R Y[3 * N];
    return term_tau<N>(b, kr, cs, Bi, T, Y);
}

#pragma nv_exec_check_disable
template <int N, typename R>
NECG_HD R term_sig(const Consts<N> &cs, const R (&T)[3 * N]) {
    R sg = cs.q[0] * T[2];
#pragma unroll
    for (int i = 1; i < N; ++i) sg += cs.q[i] * T[3 * i + 2];
    return cs.efs * sg;
}

// Energy part: returns false if B is not positive definite.
#pragma nv_exec_check_disable
template <int N, typename R, typename BA, typename KA>
NECG_HD bool term_energy(const BA &b, const KA &kr, const Consts<N> &cs, R &ov, R &tau, R &rho,
                         R &sig) {
    R Bi[tri(N)], T[3 * N];
    const bool ok = term_core<N>(b, kr, cs, Bi, T, ov);
    tau = term_tau<N>(b, kr, cs, Bi, T);
    sig = term_sig<N>(cs, T);
    // Coulomb sum (python/matel.py:162-197)
    R r = R(0.0);
#pragma unroll
    for (int q = 1; q <= N; ++q)
#pragma unroll
        for (int p = 0; p < q; ++p) {
            R a = Bi[sx(q - 1, q - 1)];
            R bv[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) bv[c] = T[3 * (q - 1) + c];
            if (p > 0) {
                a += Bi[sx(p - 1, p - 1)] - 2.0 * Bi[sx(q - 1, p - 1)];
#pragma unroll
                for (int c = 0; c < 3; ++c) bv[c] -= T[3 * (p - 1) + c];
            }
            const R bb = bv[0] * bv[0] + bv[1] * bv[1] + bv[2] * bv[2];
            R fs, D, ia, z;
            boys<false, (N > 3)>(a, bb, fs, D, ia, z);
            r += cs.cv[vidx(p, q)] * fs;
        }
    rho = r;
    return ok;
}

// Full term with bra gradient.  Fw = wgt (lam h - E ov), ovw = wgt lam ov:
// lam = 1, E = current energy gives the gradient of H - E S (the optimiser's
// combination); lam = 1, E = 0 gives dH alone; lam = 0, E = -1 gives dS alone.
// acc: accumulator with g(t) (packed dF/dA_k), d() (coefficient of A_k^-1 in
// dF/dA_k) and s(t) (dF/ds_k, n x 3), each returning a reference -- registers
// (RegAcc) or, on the device, lane-interleaved shared memory.
#pragma nv_exec_check_disable
template <int N, typename R, typename BA, typename KA, typename ACC>
NECG_HD bool term_grad(const BA &b, const KA &kr, const Consts<N> &cs, R lam, R E, R wgt, ACC &acc) {
    using KL = KetLayout<N>;
    using BL = BraLayout<N>;
    R Bi[tri(N)], T[3 * N], ov;
    const bool ok = term_core<N>(b, kr, cs, Bi, T, ov);
    const R tau = term_tau<N>(b, kr, cs, Bi, T);
    const R sig = term_sig<N>(cs, T);
    R Z[3 * N], W[tri(N)], rho;
    coulomb_grad<N>(Bi, T, cs, rho, Z, W);
    const R h = ov * (2.0 * tau + rho - sig);
    const R Fw = wgt * (lam * h - E * ov);
    const R ovw = wgt * lam * ov;
    acc.d() += 0.75 * Fw;
    // accG += Bi (ovw (6 N_l' + W) - 1.5 Fw B) Bi,  B = A_k + A_l'
    {
        const R f15 = 1.5 * Fw;
#pragma unroll
        for (int t = 0; t < tri(N); ++t)
            W[t] = ovw * (6.0 * kr[KL::Np + t] + W[t]) - f15 * (b(BL::A + t) + kr[KL::Ap + t]);
#pragma unroll
        for (int j = 0; j < N; ++j) {
            R col[N];  // column j of W Bi
#pragma unroll
            for (int a = 0; a < N; ++a) {
                R s = W[sx(a, 0)] * Bi[sx(0, j)];
#pragma unroll
                for (int k = 1; k < N; ++k) s += W[sx(a, k)] * Bi[sx(k, j)];
                col[a] = s;
            }
#pragma unroll
            for (int i = j; i < N; ++i) {
                R s = Bi[sx(i, 0)] * col[0];
#pragma unroll
                for (int a = 1; a < N; ++a) s += Bi[sx(i, a)] * col[a];
                acc.g(sx(i, j)) += s;
            }
        }
    }
    // Y = A_l' (T - S_l') ; Zk = Z' - 4 (A_l' M) Y ; Qk = Bi Zk
    R Y[3 * N];
    {
        R Dl[3 * N];
#pragma unroll
        for (int t = 0; t < 3 * N; ++t) Dl[t] = T[t] - kr[KL::Sp + t];
        symv3<N>(kr, KL::Ap, Dl, Y);
    }
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            R s = Z[3 * i + c];
#pragma unroll
            for (int k = 0; k < N; ++k) s += kr[KL::AMn4 + i * N + k] * Y[3 * k + c];
            Z[3 * i + c] = s;
        }
    R Q[3 * N];
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            R s = Bi[sx(i, 0)] * Z[c];
#pragma unroll
            for (int k = 1; k < N; ++k) s += Bi[sx(i, k)] * Z[3 * k + c];
            Q[3 * i + c] = s;
        }
    // accS += 2 ovw A_k Q - 2 Fw Y
    {
        const R o2 = 2.0 * ovw, f2 = 2.0 * Fw;
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                R s = b(BL::A + sx(i, 0)) * Q[c];
#pragma unroll
                for (int k = 1; k < N; ++k) s += b(BL::A + sx(i, k)) * Q[3 * k + c];
                acc.s(3 * i + c) += o2 * s - f2 * Y[3 * i + c];
            }
    }
    // Rk = ovw Qk - Fw/2 Dk ; accG += Rk Dk^T + Dk Rk^T,  Dk = S_k - T
    {
        const R fh = 0.5 * Fw;
#pragma unroll
        for (int t = 0; t < 3 * N; ++t) {
            const R dk = b(BL::S + t) - T[t];
            T[t] = dk;
            Q[t] = ovw * Q[t] - fh * dk;
        }
    }
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            R s = Q[3 * i] * T[3 * j] + T[3 * i] * Q[3 * j];
#pragma unroll
            for (int c = 1; c < 3; ++c) s += Q[3 * i + c] * T[3 * j + c] + T[3 * i + c] * Q[3 * j + c];
            acc.g(sx(i, j)) += s;
        }
    return ok;
}

// Both gradients of one (k, l, P) term: the bra gradient (with respect to A_k,
// s_k; weight wb) into acc, and the ket gradient with respect to the
// transformed ket (A_l' = sml^T A_l sml, s_l' = sms s_l; weight wk) through
// kout.put(f, value) / kout.add(f, value) for f in [0, tri(N) + 1 + 3N):
// packed dF/dA_l', the coefficient of A_l'^-1, dF/ds_l'.  The element is symmetric under exchanging
// bra and (transformed) ket, so the ket formulas are the bra formulas with the
// roles swapped:
//   dF/dA_l' = Fk (-Dl Dl^T - 1.5 Bi) + 0.75 Fk A_l'^-1
//              + ovk (Bi (6 A_k M A_k + W) Bi - Ql Dl^T - Dl Ql^T)
//   dF/ds_l' = 2 Fk Y + 2 ovk A_l' Ql,   Ql = Bi (Z' + 4 A_k M Y),  Dl = T - S_l'
// with Fk = wk (h - E ov), ovk = wk ov.
#pragma nv_exec_check_disable
template <int N, typename R, typename BA, typename KA, typename ACC, typename KOUT>
NECG_HD bool term_sym(const BA &b, const KA &kr, const Consts<N> &cs, R E, R wb, R wk, ACC &acc,
                      KOUT &kout) {
    using KL = KetLayout<N>;
    using BL = BraLayout<N>;
    R Bi[tri(N)], T[3 * N], ov;
    const bool ok = term_core<N>(b, kr, cs, Bi, T, ov);
    const R tau = term_tau<N>(b, kr, cs, Bi, T);
    const R sig = term_sig<N>(cs, T);
    R Z[3 * N], W[tri(N)], rho;
    coulomb_grad<N>(Bi, T, cs, rho, Z, W);
    const R phi = ov * (2.0 * tau + rho - sig) - E * ov;
    const R Fb = wb * phi, ovb = wb * ov;
    const R Fk = wk * phi, ovk = wk * ov;
    acc.d() += 0.75 * Fb;
    kout.put(tri(N), 0.75 * Fk);
    // bra: acc += Bi (ovb (6 N_l' + W) - 1.5 Fb B) Bi ; ket: Bi (ovk (6 N_k + W) - 1.5 Fk B) Bi
    {
        R Mt[tri(N)];
        const R fb = 1.5 * Fb, fk = 1.5 * Fk;
#pragma unroll
        for (int t = 0; t < tri(N); ++t)
            Mt[t] = ovb * (6.0 * kr[KL::Np + t] + W[t]) - fb * (b(BL::A + t) + kr[KL::Ap + t]);
        sandwich<N>(Bi, Mt, [&](int t, R v) { acc.g(t) += v; });
#pragma unroll
        for (int t = 0; t < tri(N); ++t)
            W[t] = ovk * (6.0 * b(BL::Nk + t) + W[t]) - fk * (b(BL::A + t) + kr[KL::Ap + t]);
        sandwich<N>(Bi, W, [&](int t, R v) { kout.put(t, v); });
    }
    // Y = A_l' (T - S_l'); Qk = Bi (Z' - 4 A_l' M Y); Ql = Bi (Z' + 4 A_k M Y) = Qk + 4 M Y
    // (the difference of the two right-hand sides is 4 B M Y and Bi B = I)
    R Dl[3 * N], Y[3 * N];
#pragma unroll
    for (int t = 0; t < 3 * N; ++t) Dl[t] = T[t] - kr[KL::Sp + t];
    symv3<N>(kr, KL::Ap, Dl, Y);
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            R s = Z[3 * i + c];
#pragma unroll
            for (int k = 0; k < N; ++k) s += kr[KL::AMn4 + i * N + k] * Y[3 * k + c];
            Z[3 * i + c] = s;
        }
    R Qk[3 * N], Ql[3 * N];
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            R s = Bi[sx(i, 0)] * Z[c];
#pragma unroll
            for (int k = 1; k < N; ++k) s += Bi[sx(i, k)] * Z[3 * k + c];
            Qk[3 * i + c] = s;
        }
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            R s = Qk[3 * i + c];
#pragma unroll
            for (int k = 0; k < N; ++k) s += cs.M4[i * N + k] * Y[3 * k + c];
            Ql[3 * i + c] = s;
        }
    // bra: acc.s += 2 ovb A_k Qk - 2 Fb Y ; ket: put 2 ovk A_l' Ql + 2 Fk Y
    {
        const R ob2 = 2.0 * ovb, fb2 = 2.0 * Fb, ok2 = 2.0 * ovk, fk2 = 2.0 * Fk;
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                R s = b(BL::A + sx(i, 0)) * Qk[c];
                R t = kr[KL::Ap + sx(i, 0)] * Ql[c];
#pragma unroll
                for (int k = 1; k < N; ++k) {
                    s += b(BL::A + sx(i, k)) * Qk[3 * k + c];
                    t += kr[KL::Ap + sx(i, k)] * Ql[3 * k + c];
                }
                acc.s(3 * i + c) += ob2 * s - fb2 * Y[3 * i + c];
                kout.put(tri(N) + 1 + 3 * i + c, ok2 * t + fk2 * Y[3 * i + c]);
            }
    }
    // bra: Rk = ovb Qk - Fb/2 Dk, acc.g += Rk Dk^T + Dk Rk^T   (Dk = S_k - T)
    // ket: Rl = ovk Ql + Fk/2 Dl, dF/dA_l' -= Rl Dl^T + Dl Rl^T
    {
        const R fbh = 0.5 * Fb, fkh = 0.5 * Fk;
#pragma unroll
        for (int t = 0; t < 3 * N; ++t) {
            const R dk = b(BL::S + t) - T[t];
            T[t] = dk;
            Qk[t] = ovb * Qk[t] - fbh * dk;
            Ql[t] = ovk * Ql[t] + fkh * Dl[t];
        }
    }
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            R s = Qk[3 * i] * T[3 * j] + T[3 * i] * Qk[3 * j];
            R t = Ql[3 * i] * Dl[3 * j] + Dl[3 * i] * Ql[3 * j];
#pragma unroll
            for (int c = 1; c < 3; ++c) {
                s += Qk[3 * i + c] * T[3 * j + c] + T[3 * i + c] * Qk[3 * j + c];
                t += Ql[3 * i + c] * Dl[3 * j + c] + Dl[3 * i + c] * Ql[3 * j + c];
            }
            acc.g(sx(i, j)) += s;
            kout.add(sx(i, j), -t);
        }
    return ok;
}

// One (k, l, P) term of the fused pass: the H element h and overlap ov (for H
// and S), and the bra and ket gradients of h and of ov kept apart -- the pass
// runs before E is known, and g = g_H - E g_S is formed once E is.  With
// Fb = wb h, ovb = wb ov (Fk, ovk with wk):
//   bra, H: the formulas of term_grad with Fw = Fb, ovw = ovb
//   bra, S: d(ov)/dA_k = ov (-Dk Dk^T - 1.5 Bi + 0.75 A_k^-1), d(ov)/ds_k = -2 ov Y
// and the ket formulas of term_sym with the same split.  The ket values of H
// and of S for field f go out together: ko.put(f, vH, vS) / ko.add(f, vH, vS).
// mid(i) is called at two points of the body (i = 1 after B, Bi, T and ov;
// i = 2 after tau and sig), for callers that synchronise warps there.  tau's
// Y = A_l' (T - S_l') goes on to the gradient formulas (it is not formed
// twice).  For n <= 3 the Coulomb sum comes before tau (and before mid(2)),
// otherwise after: the order that measured faster on a B200 for each n, since
// the values live across the Coulomb sum (Y, or Z and W) set the register
// pressure; the results are the same either way, bit for bit.
struct NoMid {
    NECG_HD void operator()(int) const {}
};
#pragma nv_exec_check_disable
template <int N, typename R, typename BA, typename KA, typename ACC, typename KOUT, typename MID = NoMid>
NECG_HD bool term_fused(const BA &b, const KA &kr, const Consts<N> &cs, R wb, R wk, ACC &accH, ACC &accS,
                        KOUT &ko, R &h_out, R &ov_out, const MID &mid = MID{}) {
    using KL = KetLayout<N>;
    using BL = BraLayout<N>;
    R Bi[tri(N)], T[3 * N], ov;
    const bool ok = term_core<N>(b, kr, cs, Bi, T, ov);
    mid(1);
    constexpr bool coulomb_first = N <= 3;
    R Z[3 * N], W[tri(N)], rho, Y[3 * N];
    if constexpr (coulomb_first) coulomb_grad<N>(Bi, T, cs, rho, Z, W);
    const R tau = term_tau<N>(b, kr, cs, Bi, T, Y);
    const R sig = term_sig<N>(cs, T);
    mid(2);
    if constexpr (!coulomb_first) coulomb_grad<N>(Bi, T, cs, rho, Z, W);
    const R h = ov * (2.0 * tau + rho - sig);
    h_out = h;
    ov_out = ov;
    const R Fb = wb * h, ovb = wb * ov;
    const R Fk = wk * h, ovk = wk * ov;
    accH.d() += 0.75 * Fb;
    accS.d() += 0.75 * ovb;
    ko.put(tri(N), 0.75 * Fk, 0.75 * ovk);
    // Bi (ovb (6 N_l' + W) - 1.5 Fb B) Bi = Bi ovb (6 N_l' + W) Bi - 1.5 Fb Bi, since
    // Bi B Bi = Bi (and the same for the ket)
    {
        R Mt[tri(N)];
        const R fb = 1.5 * Fb, fk = 1.5 * Fk, sb = 1.5 * ovb, sk = 1.5 * ovk;
#pragma unroll
        for (int t = 0; t < tri(N); ++t) Mt[t] = ovb * (6.0 * kr[KL::Np + t] + W[t]);
        sandwich_seeded<N>(Bi, Mt, [&](int t) { return accH.g(t) - fb * Bi[t]; },
                           [&](int t, R v) { accH.g(t) = v; });
#pragma unroll
        for (int t = 0; t < tri(N); ++t) W[t] = ovk * (6.0 * b(BL::Nk + t) + W[t]);
        // S parts: Bi (-1.5 ov B) Bi = -1.5 ov Bi
        sandwich_seeded<N>(Bi, W, [&](int t) { return -(fk * Bi[t]); },
                           [&](int t, R v) { ko.put(t, v, -(sk * Bi[t])); });
#pragma unroll
        for (int t = 0; t < tri(N); ++t) accS.g(t) = accS.g(t) - sb * Bi[t];
    }
    // Qk = Bi (Z' - 4 A_l' M Y); Ql = Bi (Z' + 4 A_k M Y) = Qk + 4 M Y (the
    // difference of the two right-hand sides is 4 B M Y and Bi B = I)
    R Dl[3 * N];
#pragma unroll
    for (int t = 0; t < 3 * N; ++t) Dl[t] = T[t] - kr[KL::Sp + t];
    // the ket and bra matrices below are read once per element and used for
    // the three columns; each output's products are summed in the same order
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const R a = kr[KL::AMn4 + i * N + k];
#pragma unroll
            for (int c = 0; c < 3; ++c) Z[3 * i + c] += a * Y[3 * k + c];
        }
    R Qk[3 * N], Ql[3 * N];
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            R s = Bi[sx(i, 0)] * Z[c];
#pragma unroll
            for (int k = 1; k < N; ++k) s += Bi[sx(i, k)] * Z[3 * k + c];
            Qk[3 * i + c] = s;
        }
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            R s = Qk[3 * i + c];
#pragma unroll
            for (int k = 0; k < N; ++k) s += cs.M4[i * N + k] * Y[3 * k + c];
            Ql[3 * i + c] = s;
        }
    // H: bra s += 2 ovb A_k Qk - 2 Fb Y, ket 2 ovk A_l' Ql + 2 Fk Y ; S: -2 ovb Y, +2 ovk Y
    {
        const R ob2 = 2.0 * ovb, fb2 = 2.0 * Fb, ok2 = 2.0 * ovk, fk2 = 2.0 * Fk;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            R s[3], t[3];
            {
                const R a = b(BL::A + sx(i, 0)), ap = kr[KL::Ap + sx(i, 0)];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    s[c] = a * Qk[c];
                    t[c] = ap * Ql[c];
                }
            }
#pragma unroll
            for (int k = 1; k < N; ++k) {
                const R a = b(BL::A + sx(i, k)), ap = kr[KL::Ap + sx(i, k)];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    s[c] += a * Qk[3 * k + c];
                    t[c] += ap * Ql[3 * k + c];
                }
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const R y = Y[3 * i + c];
                accH.s(3 * i + c) = (accH.s(3 * i + c) - fb2 * y) + ob2 * s[c];
                accS.s(3 * i + c) = accS.s(3 * i + c) - ob2 * y;
                ko.put(tri(N) + 1 + 3 * i + c, ok2 * t[c] + fk2 * y, ok2 * y);
            }
        }
    }
    // H: Rk = ovb Qk - Fb/2 Dk, acc += Rk Dk^T + Dk Rk^T ; Rl = ovk Ql + Fk/2 Dl, ket -= Rl Dl^T + Dl Rl^T
    // S: bra -= ovb Dk Dk^T, ket -= ovk Dl Dl^T
    {
        const R fbh = 0.5 * Fb, fkh = 0.5 * Fk;
#pragma unroll
        for (int t = 0; t < 3 * N; ++t) {
            const R dk = b(BL::S + t) - T[t];
            T[t] = dk;
            Qk[t] = ovb * Qk[t] - fbh * dk;
            Ql[t] = ovk * Ql[t] + fkh * Dl[t];
        }
    }
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            R s = accH.g(sx(i, j));  // the products fuse into the accumulator
            R t = Ql[3 * i] * Dl[3 * j] + Dl[3 * i] * Ql[3 * j];
            R dd = T[3 * i] * T[3 * j], ee = Dl[3 * i] * Dl[3 * j];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                s += Qk[3 * i + c] * T[3 * j + c];
                s += T[3 * i + c] * Qk[3 * j + c];
            }
#pragma unroll
            for (int c = 1; c < 3; ++c) {
                t += Ql[3 * i + c] * Dl[3 * j + c] + Dl[3 * i + c] * Ql[3 * j + c];
                dd += T[3 * i + c] * T[3 * j + c];
                ee += Dl[3 * i + c] * Dl[3 * j + c];
            }
            accH.g(sx(i, j)) = s;
            accS.g(sx(i, j)) = accS.g(sx(i, j)) - ovb * dd;
            ko.add(sx(i, j), -t, -(ovk * ee));
        }
    return ok;
}

// One term of the dipole element of python/rrms.py:21-120 for the bra record
// (k, Pe) and the ket record (l, P) (both in KetLayout: symmetry applied to both
// sides): B = A_k'' + A_l', T = Bi (A_k'' s_k'' + A_l' s_l') (rrms's st), and
// ov = sqrt(8^n) (|L_k| |L_l| / |B|)^{3/2} exp(<e, T> - i1 - i2).  rrms returns
// (ov, T[n1] ov).  Returns false if B is not positive definite.
#pragma nv_exec_check_disable
template <int N, typename R, typename KA, typename KB>
NECG_HD bool term_dipole(const KA &kb, const KB &kr, const Consts<N> &cs, R (&T)[3 * N], R &ov) {
    using KL = KetLayout<N>;
    R Bi[tri(N)], prinv;
    bool ok;
    {
        R B[tri(N)];
#pragma unroll
        for (int t = 0; t < tri(N); ++t) B[t] = kb[KL::Ap + t] + kr[KL::Ap + t];
        ok = chol_inverse<N>(B, Bi, prinv);
    }
    R e[3 * N];
#pragma unroll
    for (int t = 0; t < 3 * N; ++t) e[t] = kb[KL::ASp + t] + kr[KL::ASp + t];
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            R s = Bi[sx(i, 0)] * e[c];
#pragma unroll
            for (int k = 1; k < N; ++k) s += Bi[sx(i, k)] * e[3 * k + c];
            T[3 * i + c] = s;
        }
    R i3 = e[0] * T[0];
#pragma unroll
    for (int t = 1; t < 3 * N; ++t) i3 += e[t] * T[t];
    const R p3 = prinv * prinv * prinv;
    ov = cs.sqrt8n * kb[KL::pre] * kr[KL::pre] * p3 * exp(i3 - kb[KL::i2] - kr[KL::i2]);
    return ok;
}

}  // namespace necg
