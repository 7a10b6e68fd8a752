// necg_lanes.cuh -- per-thread bodies of the kernels, shared by the CUDA
// kernels (R = double, device accessors) and by the host-side test emulator
// (R = a value-carrying scalar, host accessors), so that the emulator exercises
// exactly the index arithmetic, loop bounds and reductions the kernels run.
#pragma once
#include "necg_math.cuh"

namespace necg {

NECG_HD double val(double x) { return x; }

// Unpack vech(L) (python/matel.py:59-66: column-major lower triangle) into a
// packed-lower row-major array.
template <int N> NECG_HD void unpack_L(const double *blk, double (&L)[tri(N)]) {
    int idx = 0;
#pragma unroll
    for (int j = 0; j < N; ++j)
#pragma unroll
        for (int i = j; i < N; ++i) L[sx(i, j)] = blk[idx++];
}

// A = L L^T (packed)
template <int N> NECG_HD void llt(const double (&L)[tri(N)], double (&A)[tri(N)]) {
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

// A M (full), A M A (packed) and tr(M A)
template <int N>
NECG_HD void mass_products(const double (&A)[tri(N)], const double *M, double (&AM)[N * N],
                           double (&AMA)[tri(N)], double &tMA) {
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

// Bra record of basis k (structure of arrays, field f at f*K + k).
template <int N>
NECG_HD void prep_bra_one(const double *iv, int K, const Consts<N> &cs, double *bra, int k) {
    using BL = BraLayout<N>;
    constexpr int blk = tri(N) + 3 * N;
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
    dl = ::fabs(dl);
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
    bra[BL::pre * KK + k] = dl * ::sqrt(dl);
    bra[BL::tMA * KK + k] = tMA;
#pragma unroll
    for (int t = 0; t < tri(N); ++t) bra[(BL::L + t) * KK + k] = L[t];
}

// Ket record of (l, P) = id / nst, id % nst: python/matel.py:76-87
// (al <- sml^T al sml, st2 <- sms st2) plus the data the tiles reuse.
template <int N>
NECG_HD void prep_ket_one(const double *iv, const double *C, int nst, const Consts<N> &cs,
                          const double *sml, const double *sms, const double *scvv, double *ket,
                          int id, const int *pinv = nullptr) {
    using KL = KetLayout<N>;
    constexpr int blk = tri(N) + 3 * N;
    const int l = id / nst, P = id - l * nst;
    const double *b = iv + (size_t)l * blk;
    double L[tri(N)], A[tri(N)];
    unpack_L<N>(b, L);
    llt<N>(L, A);
    const double *pm = sml + (size_t)P * N * N;
    double Apm[N * N];  // A pm
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < N; ++k) s += A[sx(i, k)] * pm[k * N + j];
            Apm[i * N + j] = s;
        }
    double Ap[tri(N)];  // pm^T A pm
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < N; ++k) s += pm[k * N + i] * Apm[k * N + j];
            Ap[sx(i, j)] = s;
        }
    const double *sm = sms + (size_t)P * 9 * N * N;  // general 3n x 3n shift map
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
    dl = ::fabs(dl);
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
    for (int t = 0; t < N * N; ++t) o[KL::AMn4 + t] = -4.0 * AM[t];
    o[KL::i2] = i2;
    o[KL::pre] = dl * ::sqrt(dl);
    o[KL::tMA] = tMA;
    o[KL::w] = scvv[P];
    o[KL::wC] = C ? 2.0 * scvv[P] * C[l] : 0.0;
    o[KL::winv] = pinv ? scvv[pinv[P]] : 0.0;
    if (KL::size > KL::winv + 1) o[KL::winv + 1] = 0.0;
}

// Energy tile lane: bra k against kets l in [l0, lend) (lend <= k + 1), all P.
// Writes H, S (and Kin, Pot when non-null) symmetrically.  Returns status
// flags (1: a pair not positive definite, 2: non-finite) and the first pair.
template <int N, typename R, typename BA, typename KB>
NECG_HD int energy_lane(const BA &b, const KB &ket, int k, int l0, int lend, int K, int nst,
                        const Consts<N> &cs, double *H, double *S, double *Kin, double *Pot,
                        int &bad_pair) {
    using KL = KetLayout<N>;
    int flags = 0;
    for (int l = l0; l < lend; ++l) {
        R h = R(0.0), s = R(0.0), tkin = R(0.0), tpot = R(0.0);
        bool ok = true;
        for (int P = 0; P < nst; ++P) {
            const auto kr = ket.at(((size_t)l * nst + P) * KL::size);
            R ov, tau, rho, sig;
            ok = term_energy<N>(b, kr, cs, ov, tau, rho, sig) && ok;
            const R wov = kr[KL::w] * ov;
            const R t2 = 2.0 * tau;
            h += wov * (t2 + rho - sig);
            s += wov;
            tkin += wov * t2;
            tpot += wov * rho;
        }
        const double hv = val(h), sv = val(s);
        int fl = ok ? 0 : 1;
        if (!isfinite(hv) || !isfinite(sv)) fl |= 2;
        if (fl && !flags) bad_pair = k * K + l;
        flags |= fl;
        H[(size_t)k * K + l] = hv;
        H[(size_t)l * K + k] = hv;
        S[(size_t)k * K + l] = sv;
        S[(size_t)l * K + k] = sv;
        if (Kin) {
            Kin[(size_t)k * K + l] = val(tkin);
            Kin[(size_t)l * K + k] = val(tkin);
        }
        if (Pot) {
            Pot[(size_t)k * K + l] = val(tpot);
            Pot[(size_t)l * K + k] = val(tpot);
        }
    }
    return flags;
}

// Partial-buffer stride (doubles per basis function): dF/dA_k packed, the
// coefficient of A_k^-1 in dF/dA_k, dF/ds_k.
template <int N> struct Part {
    static constexpr int G = 0;
    static constexpr int D = tri(N);
    static constexpr int S = D + 1;
    static constexpr int size = S + 3 * N;
};

// Gradient tile lane: bra k against kets l in [l0, l1), all P, weights
// wC(l, P) = 2 scvv[P] C_l; writes the partial to part[f * stride] (f < Part::size).
template <int N, typename R, typename BA, typename KB, typename ACC>
NECG_HD bool grad_lane(const BA &b, const KB &ket, int l0, int l1, int nst, const Consts<N> &cs,
                       R lam, R E, double *part, size_t stride, ACC &acc) {
    using KL = KetLayout<N>;
    using PL = Part<N>;
    acc.zero();
    bool ok = true;
    for (int l = l0; l < l1; ++l)
        for (int P = 0; P < nst; ++P) {
            const auto kr = ket.at(((size_t)l * nst + P) * KL::size);
            ok = term_grad<N>(b, kr, cs, lam, E, R(kr[KL::wC]), acc) && ok;
        }
#pragma unroll
    for (int t = 0; t < tri(N); ++t) part[(PL::G + t) * stride] = val(acc.g(t));
    part[PL::D * stride] = val(acc.d());
#pragma unroll
    for (int t = 0; t < 3 * N; ++t) part[(PL::S + t) * stride] = val(acc.s(t));
    return ok;
}

template <int N, typename R, typename BA, typename KB>
NECG_HD bool grad_lane(const BA &b, const KB &ket, int l0, int l1, int nst, const Consts<N> &cs,
                       R lam, R E, double *part, size_t stride) {
    RegAcc<N, R> acc;
    return grad_lane<N, R>(b, ket, l0, l1, nst, cs, lam, E, part, stride, acc);
}

// Map an A-space gradient dF/dA = G + D A^-1 (G packed symmetric, D the
// scalar coefficient of A^-1) and dF/ds = gS to the reference's parameter
// block [vech(dF/dL), dF/ds]: dF/dL = 2 (G + D A^-1) L = 2 G L + 2 D L^-T, whose
// lower triangle is 2 (G L)_ij for i > j and 2 (G L)_ii + 2 D / L_ii on the
// diagonal.  out[blk] scaled by sc.
template <int N>
NECG_HD bool a_to_vech(const double (&G)[tri(N)], double D, const double (&gS)[3 * N],
                       const double (&L)[tri(N)], double sc, double *out) {
    int idx = 0;
    bool fin = true;
#pragma unroll
    for (int j = 0; j < N; ++j)
#pragma unroll
        for (int i = j; i < N; ++i) {
            double s = 0.0;  // (G L)_ij = sum_{a >= j} G_ia L_aj
#pragma unroll
            for (int a = j; a < N; ++a) s += G[sx(i, a)] * L[sx(a, j)];
            s *= 2.0;
            if (i == j) s += 2.0 * D / L[sx(i, i)];
            const double v = sc * s;
            fin = fin && isfinite(v);
            out[idx++] = v;
        }
#pragma unroll
    for (int t = 0; t < 3 * N; ++t) {
        const double v = sc * gS[t];
        fin = fin && isfinite(v);
        out[tri(N) + t] = v;
    }
    return fin;
}

// Sum the nlc partials of basis k and write its GRADA block scaled by sc.
template <int N>
NECG_HD bool grad_reduce_one(const double *part, int nlc, int K, const double *bra, double sc,
                             double *g, int k) {
    using BL = BraLayout<N>;
    using PL = Part<N>;
    constexpr int blk = tri(N) + 3 * N;
    double G[tri(N)], gS[3 * N], D = 0.0, L[tri(N)];
#pragma unroll
    for (int t = 0; t < tri(N); ++t) G[t] = 0.0;
#pragma unroll
    for (int t = 0; t < 3 * N; ++t) gS[t] = 0.0;
    for (int lc = 0; lc < nlc; ++lc) {
        const double *p = part + (size_t)lc * PL::size * K + k;
#pragma unroll
        for (int t = 0; t < tri(N); ++t) G[t] += p[(size_t)(PL::G + t) * K];
        D += p[(size_t)PL::D * K];
#pragma unroll
        for (int t = 0; t < 3 * N; ++t) gS[t] += p[(size_t)(PL::S + t) * K];
    }
#pragma unroll
    for (int t = 0; t < tri(N); ++t) L[t] = bra[(BL::L + t) * (size_t)K + k];
    return a_to_vech<N>(G, D, gS, L, sc, g + (size_t)k * blk);
}

// One matel term (python/matel.py:28-210): out = (ov, tk, ert, zht).
template <int N, typename R, typename BA, typename KR>
NECG_HD bool matel_one(const BA &b, const KR &kr, const Consts<N> &cs, double *out) {
    R ov, tau, rho, sig;
    const bool ok = term_energy<N>(b, kr, cs, ov, tau, rho, sig);
    out[0] = val(ov);
    out[1] = val(2.0 * ov * tau);
    out[2] = val(ov * rho);
    out[3] = val(ov * sig);
    return ok;
}

// One gradel term (python/gradel.py:27-392): dH and dS with respect to the bra
// block, doubled when ii == jj (python/gradel.py:388-390).
template <int N, typename R, typename BA, typename KR>
NECG_HD bool gradel_one(const BA &b, const KR &kr, const Consts<N> &cs, const double (&L)[tri(N)],
                        bool diag, double *tgvl, double *tgvls) {
    bool ok = true;
#pragma unroll
    for (int which = 0; which < 2; ++which) {
        RegAcc<N, R> acc;
        acc.zero();
        // which 0: dH (lam 1, E 0); which 1: dS (lam 0, E -1)
        ok = term_grad<N>(b, kr, cs, R(which == 0 ? 1.0 : 0.0), R(which == 0 ? 0.0 : -1.0), R(1.0), acc) && ok;
        double G[tri(N)], gS[3 * N];
#pragma unroll
        for (int q = 0; q < tri(N); ++q) G[q] = val(acc.g(q));
#pragma unroll
        for (int q = 0; q < 3 * N; ++q) gS[q] = val(acc.s(q));
        a_to_vech<N>(G, val(acc.d()), gS, L, diag ? 2.0 : 1.0, which == 0 ? tgvl : tgvls);
    }
    return ok;
}

// Energy tiles over the lower triangle: tile (kb, lc) covers bra k in
// [32 kb, 32 kb + 32) and kets l in [lc LC, lc LC + LC) with l <= k; a tile
// exists when lc LC <= 32 kb + 31 and lc LC < K.
NECG_HD int energy_tile_count(int K, int LC) {
    int n = 0;
    for (int kb = 0; kb * 32 < K; ++kb) {
        const int kmax = kb * 32 + 31;
        const int last = kmax < K - 1 ? kmax : K - 1;
        n += last / LC + 1;
    }
    return n;
}

// Sparse linear map taking a ket gradient from P's transformed frame to the
// basis function's own frame: dF/dA_l = sml dF/dA_l' sml^T (packed), the A^-1
// coefficient unchanged, dF/ds_l = sms^T dF/ds_l'.  Entry (P, f): cnt values
// at src/coef[(P * PS + f) * maxnz + i].
struct KetMap {
    const int *cnt, *src;
    const double *coef;
    int maxnz;
};

NECG_HD double ket_map_apply(const KetMap &m, int P, int f, int PS, const double *in) {
    const int e = P * PS + f;
    const int n = m.cnt[e];
    double v = 0.0;
    for (int i = 0; i < n; ++i) v += m.coef[(size_t)e * m.maxnz + i] * in[m.src[(size_t)e * m.maxnz + i]];
    return v;
}

// The same map applied to two inputs (the H and S ket gradients), reading the
// map entries once.
NECG_HD void ket_map_apply2(const KetMap &m, int P, int f, int PS, const double *in0, const double *in1,
                            double &out0, double &out1) {
    const int e = P * PS + f;
    const int n = m.cnt[e];
    double v0 = 0.0, v1 = 0.0;
    for (int i = 0; i < n; ++i) {
        const double c = m.coef[(size_t)e * m.maxnz + i];
        const int s = m.src[(size_t)e * m.maxnz + i];
        v0 += c * in0[s];
        v1 += c * in1[s];
    }
    out0 = v0;
    out1 = v1;
}

// Lane ranges of the two tile kinds (used by the kernels and the emulator).
// Energy: tile (kb, lc) -> bra k = 32 kb + lane, kets [l0, lend); false if idle.
NECG_HD bool energy_lane_range(int kb, int lc, int lane, int LC, int K, int &k, int &l0, int &lend) {
    k = kb * 32 + lane;
    l0 = lc * LC;
    if (k >= K || l0 > k) return false;
    lend = l0 + LC < K ? l0 + LC : K;
    if (lend > k + 1) lend = k + 1;
    return true;
}
// Gradient: warp w -> (kb = w % nkb, lc = w / nkb), bra k = 32 kb + lane,
// kets [l0, l1); false if idle.
NECG_HD bool grad_lane_range(int w, int lane, int nkb, int LC, int K, int &k, int &lc, int &l0,
                             int &l1) {
    const int kb = w % nkb;
    lc = w / nkb;
    k = kb * 32 + lane;
    if (k >= K) return false;
    l0 = lc * LC;
    l1 = l0 + LC < K ? l0 + LC : K;
    return true;
}

}  // namespace necg
