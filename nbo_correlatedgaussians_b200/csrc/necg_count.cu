// necg_count.cu -- algorithmic FP64 operation count of one (k, l, P) term.
//
// The term templates of necg_math.cuh are instantiated on the host with a
// counting scalar: every add, subtract and multiply counts 1 (so a fused
// multiply-add counts 2), every division, square root, reciprocal square root
// and exponential counts 1 in a separate "special" tally.  Negation and
// comparisons are free.  The count follows the Pade branch of F0 (the branch
// all pairs of the synthetic workloads take) and excludes the per-basis and
// per-(l, P) preparation, which is amortised over K terms.
#include <math.h>
#include <stdlib.h>

#include <vector>

#include "necg_math.cuh"
#include "necg_hostscalar.cuh"
#include "../../include/necg.h"

namespace necg {

// Build one bra record (K = 1) and one ket record from a well-conditioned pair.
template <int N> void host_records(std::vector<double> &bra, std::vector<double> &ket) {
    using BL = BraLayout<N>;
    using KL = KetLayout<N>;
    bra.assign(BL::size, 0.0);
    ket.assign(KL::size, 0.0);
    double A[tri(N)], Ap[tri(N)];
    for (int i = 0; i < N; ++i)
        for (int j = 0; j <= i; ++j) {
            A[sx(i, j)] = (i == j) ? 1.0 + 0.1 * i : 0.05;
            Ap[sx(i, j)] = (i == j) ? 0.8 + 0.2 * i : -0.03;
        }
    for (int t = 0; t < tri(N); ++t) {
        bra[BL::A + t] = A[t];
        bra[BL::Nk + t] = 0.5 * A[t];
        bra[BL::L + t] = A[t];
        ket[KL::Ap + t] = Ap[t];
        ket[KL::Np + t] = 0.5 * Ap[t];
    }
    for (int t = 0; t < 3 * N; ++t) {
        bra[BL::S + t] = 0.01 * (t + 1);
        bra[BL::AS + t] = 0.02 * (t + 1);
        ket[KL::Sp + t] = -0.01 * (t + 2);
        ket[KL::ASp + t] = -0.015 * (t + 2);
    }
    for (int t = 0; t < N * N; ++t) ket[KL::AMn4 + t] = -0.04 * t;
    bra[BL::i1] = 0.01;
    bra[BL::pre] = 1.0;
    bra[BL::tMA] = 2.0;
    ket[KL::i2] = 0.02;
    ket[KL::pre] = 1.0;
    ket[KL::tMA] = 1.0;
    ket[KL::w] = 1.0;
    ket[KL::wC] = 1.0;
    ket[KL::winv] = 1.0;
}

// Ket-side output of one term: put stores, add accumulates (one add counted).
struct CountRow {
    double r[64];
    void put(int f, CD v) { r[f] = v.v; }
    void add(int f, CD v) {
        r[f] += v.v;
        ++count_ctx().flops;
    }
};
// The fused pass's ket output: the H and S values of one field together.
struct CountRow2 {
    CountRow h, s;
    void put(int f, CD vh, CD vs) {
        h.put(f, vh);
        s.put(f, vs);
    }
    void add(int f, CD vh, CD vs) {
        h.add(f, vh);
        s.add(f, vs);
    }
};

template <int N> void count_term(int which, long long &flops, long long &special) {
    std::vector<double> bra, ket;
    host_records<N>(bra, ket);
    Consts<N> cs;
    for (int i = 0; i < N * N; ++i) cs.M[i] = (i % (N + 1) == 0) ? 0.5 : 0.01;
    cs.derive();
    for (int t = 0; t < tri(N); ++t) cs.cv[t] = 1.0;
    for (int i = 0; i < N; ++i) cs.q[i] = -1.0;
    cs.efs = 1e-4;
    cs.sqrt8n = ::sqrt(::pow(8.0, N));
    HostBra b{bra.data(), 1};
    HostKet kr{ket.data()};
    count_ctx() = CountCtx();
    if (which == 0) {
        CD ov, tau, rho, sig;
        term_energy<N>(b, kr, cs, ov, tau, rho, sig);
        // the energy kernel's per-term accumulation: h, s, kinetic, potential
        CD w(1.0), h(0.0), s(0.0);
        h += w * ov * (2.0 * tau + rho - sig);
        s += w * ov;
    } else if (which == 1) {
        RegAcc<N, CD> acc;
        acc.zero();
        count_ctx() = CountCtx();  // zeroing the accumulators is not part of a term
        term_grad<N>(b, kr, cs, CD(1.0), CD(0.5), CD(1.0), acc);
    } else if (which == 2) {
        RegAcc<N, CD> acc;
        acc.zero();
        CountRow ko;
        count_ctx() = CountCtx();
        // the ket row's warp column sum and frame map are counted per (l, P),
        // not per term: they are amortised over the 32 bras of a tile
        term_sym<N>(b, kr, cs, CD(0.5), CD(1.0), CD(1.0), acc, ko);
    } else {
        RegAcc<N, CD> aH, aS;
        aH.zero();
        aS.zero();
        CountRow2 ko;
        count_ctx() = CountCtx();
        CD h, ov, hs(0.0), ss(0.0), w(1.0);
        term_fused<N>(b, kr, cs, CD(1.0), CD(1.0), aH, aS, ko, h, ov);
        hs += w * h;  // the pass's sums of w_P h and w_P ov over P
        ss += w * ov;
    }
    flops = count_ctx().flops;
    special = count_ctx().special;
}

}  // namespace necg

extern "C" long long necg_term_flops(int n, int which, long long *special) {
    long long f = 0, s = 0;
    switch (n) {
    case 1: necg::count_term<1>(which, f, s); break;
    case 2: necg::count_term<2>(which, f, s); break;
    case 3: necg::count_term<3>(which, f, s); break;
    case 4: necg::count_term<4>(which, f, s); break;
    case 5: necg::count_term<5>(which, f, s); break;
    case 6: necg::count_term<6>(which, f, s); break;
    default: return -1;
    }
    if (special) *special = s;
    return f + s;
}
