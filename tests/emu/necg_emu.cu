// necg_emu.cu -- TEST INFRASTRUCTURE: runs the kernels' per-thread bodies
// (nbo_correlatedgaussians_b200/csrc/necg_lanes.cuh) on the host, lane by lane
// and tile by tile in the kernels' own order, so the CPU test suite can check
// the device algorithm (index arithmetic, tile bounds, reductions, A-space to
// vech mapping) against the oracle without a GPU.  Never linked into the
// product library.
#include <math.h>
#include <string.h>

#include <vector>

#include "../../nbo_correlatedgaussians_b200/csrc/necg_hostscalar.cuh"
#include "../../nbo_correlatedgaussians_b200/csrc/necg_lanes.cuh"

using namespace necg;

namespace {

template <int N> Consts<N> consts(const double *mass, const double *ncv, double efs) {
    Consts<N> c;
    for (int i = 0; i < N * N; ++i) c.M[i] = mass[i];
    for (int q = 1; q <= N; ++q)
        for (int p = 0; p < q; ++p) c.cv[vidx(p, q)] = 2.0 * ncv[p] * ncv[q] / NECG_SQRT_PI;
    for (int i = 0; i < N; ++i) c.q[i] = ncv[i + 1];
    c.efs = efs;
    c.sqrt8n = ::sqrt(::pow(8.0, N));
    return c;
}

struct Args {
    int nst, K;
    double efs;
    const double *mass, *ncv, *scvv, *sml, *sms;
};

template <int N>
void prep(const Args &a, const double *iv, const double *C, std::vector<double> &bra,
          std::vector<double> &ket, const Consts<N> &cs) {
    bra.assign((size_t)BraLayout<N>::size * a.K, 0.0);
    ket.assign((size_t)KetLayout<N>::size * a.K * a.nst, 0.0);
    for (int k = 0; k < a.K; ++k) prep_bra_one<N>(iv, a.K, cs, bra.data(), k);
    for (int id = 0; id < a.K * a.nst; ++id)
        prep_ket_one<N>(iv, C, a.nst, cs, a.sml, a.sms, a.scvv, ket.data(), id);
}

template <int N>
int outprod(const Args &a, const double *x, int LCe, int LCg, double *f, double *g, double *H,
            double *S) {
    const int K = a.K, nst = a.nst;
    const size_t siv = (size_t)K * (tri(N) + 3 * N);
    const double *iv = x, *C = x + siv;
    Consts<N> cs = consts<N>(a.mass, a.ncv, a.efs);
    std::vector<double> bra, ket;
    prep<N>(a, iv, C, bra, ket, cs);
    int flags = 0;
    // energy tiles in the order of the device tile list
    for (int kb = 0; kb * 32 < K; ++kb)
        for (int lc = 0; lc * LCe <= kb * 32 + 31 && lc * LCe < K; ++lc)
            for (int lane = 0; lane < 32; ++lane) {
                int k, l0, lend, bad = 0;
                if (!energy_lane_range(kb, lc, lane, LCe, K, k, l0, lend)) continue;
                flags |= energy_lane<N, CD>(HostBra{bra.data() + k, (size_t)K},
                                            HostKetBase{ket.data()}, k, l0, lend, K, nst, cs, H, S,
                                            nullptr, nullptr, bad);
            }
    // rows + finalize
    std::vector<double> rh(K), rs(K);
    for (int i = 0; i < K; ++i) {
        double h = 0.0, s = 0.0;
        for (int j = 0; j < K; ++j) {
            h += H[(size_t)i * K + j] * C[j];
            s += S[(size_t)i * K + j] * C[j];
        }
        rh[i] = h;
        rs[i] = s;
    }
    double cHc = 0.0, cSc = 0.0;
    for (int i = 0; i < K; ++i) {
        cHc += C[i] * rh[i];
        cSc += C[i] * rs[i];
    }
    const double E = cHc / cSc, norm = 1.0 / cSc;
    *f = E;
    for (int i = 0; i < K; ++i) g[siv + i] = 2.0 * norm * (rh[i] - E * rs[i]);
    // gradient tiles
    const int nkb = (K + 31) / 32, nlc = (K + LCg - 1) / LCg;
    std::vector<double> part((size_t)Part<N>::size * K * nlc, 0.0);
    for (int w = 0; w < nkb * nlc; ++w)
        for (int lane = 0; lane < 32; ++lane) {
            int k, lc, l0, l1;
            if (!grad_lane_range(w, lane, nkb, LCg, K, k, lc, l0, l1)) continue;
            if (!grad_lane<N, CD>(HostBra{bra.data() + k, (size_t)K}, HostKetBase{ket.data()}, l0, l1,
                                  nst, cs, CD(1.0), CD(E), part.data() + (size_t)lc * Part<N>::size * K + k,
                                  (size_t)K))
                flags |= 1;
        }
    for (int k = 0; k < K; ++k)
        if (!grad_reduce_one<N>(part.data(), nlc, K, bra.data(), norm * C[k], g, k)) flags |= 2;
    return flags;
}

template <int N>
int elements(const Args &a, const double *iv, int nterms, const int *terms, double *mat,
             double *tg, double *tgs) {
    constexpr int blk = tri(N) + 3 * N;
    Consts<N> cs = consts<N>(a.mass, a.ncv, a.efs);
    std::vector<double> bra, ket;
    prep<N>(a, iv, nullptr, bra, ket, cs);
    int flags = 0;
    for (int t = 0; t < nterms; ++t) {
        const int stf = terms[3 * t] - 1, ii = terms[3 * t + 1] - 1, jj = terms[3 * t + 2] - 1;
        const HostKet kr{ket.data() + ((size_t)jj * a.nst + stf) * KetLayout<N>::size};
        const HostBra b{bra.data() + ii, (size_t)a.K};
        if (!matel_one<N, CD>(b, kr, cs, mat + 4 * t)) flags |= 1;
        double L[tri(N)];
        for (int q = 0; q < tri(N); ++q) L[q] = bra[(BraLayout<N>::L + q) * (size_t)a.K + ii];
        if (!gradel_one<N, CD>(b, kr, cs, L, ii == jj, tg + (size_t)t * blk, tgs + (size_t)t * blk))
            flags |= 1;
    }
    return flags;
}

}  // namespace

#define EMU_DISPATCH(n, expr)               \
    switch (n) {                            \
    case 1: { constexpr int N = 1; return expr; } \
    case 2: { constexpr int N = 2; return expr; } \
    case 3: { constexpr int N = 3; return expr; } \
    case 4: { constexpr int N = 4; return expr; } \
    case 5: { constexpr int N = 5; return expr; } \
    case 6: { constexpr int N = 6; return expr; } \
    default: return -1;                     \
    }

extern "C" int emu_outprod(int n, int nst, int K, double efs, const double *mass, const double *ncv,
                           const double *scvv, const double *sml, const double *sms, const double *x,
                           int lc_e, int lc_g, double *f, double *g, double *H, double *S) {
    Args a{nst, K, efs, mass, ncv, scvv, sml, sms};
    EMU_DISPATCH(n, (outprod<N>(a, x, lc_e, lc_g, f, g, H, S)));
}

extern "C" int emu_elements(int n, int nst, int K, double efs, const double *mass, const double *ncv,
                            const double *scvv, const double *sml, const double *sms, const double *iv,
                            int nterms, const int *terms, double *mat, double *tg, double *tgs) {
    Args a{nst, K, efs, mass, ncv, scvv, sml, sms};
    EMU_DISPATCH(n, (elements<N>(a, iv, nterms, terms, mat, tg, tgs)));
}
