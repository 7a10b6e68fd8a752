// necg_emu.cu -- TEST INFRASTRUCTURE: runs the kernels' per-thread bodies
// (nbo_correlatedgaussians_b200/csrc/necg_lanes.cuh) on the host, lane by lane
// and tile by tile in the kernels' own order, so the CPU test suite can check
// the device algorithm (index arithmetic, tile bounds, reductions, A-space to
// vech mapping) against the oracle without a GPU.  Never linked into the
// product library.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../nbo_correlatedgaussians_b200/csrc/necg_hostscalar.cuh"
#include "../../nbo_correlatedgaussians_b200/csrc/necg_lanes.cuh"

using namespace necg;

namespace {

template <int N> Consts<N> consts(const double *mass, const double *ncv, double efs) {
    Consts<N> c;
    for (int i = 0; i < N * N; ++i) c.M[i] = mass[i];
    c.derive();
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

// Host mirror of the symmetric gradient pass (gsym_kernel + gsym_sum_kernel):
// same tiles, same per-lane term_sym, the warp's column sums taken in lane
// order, the same ket-frame map.
struct HostMap {
    std::vector<int> cnt, src;
    std::vector<double> coef;
    int maxnz = 1;
    std::vector<int> pinv;
    bool ok = false;
};

template <int N> HostMap build_map(const Args &a) {
    HostMap hm;
    const int n = N, nst = a.nst, m = 3 * n, T = tri(N), PS = T + 1 + m;
    hm.pinv.assign(nst, -1);
    for (int p = 0; p < nst; ++p)
        for (int q = 0; q < nst && hm.pinv[p] < 0; ++q) {
            bool ok = true;
            for (int i = 0; i < n && ok; ++i)
                for (int j = 0; j < n && ok; ++j) {
                    double s = 0.0;
                    for (int k = 0; k < n; ++k) s += a.sml[p * n * n + i * n + k] * a.sml[q * n * n + k * n + j];
                    ok = fabs(s - (i == j)) < 1e-12;
                }
            for (int i = 0; i < m && ok; ++i)
                for (int j = 0; j < m && ok; ++j) {
                    double s = 0.0;
                    for (int k = 0; k < m; ++k) s += a.sms[p * m * m + i * m + k] * a.sms[q * m * m + k * m + j];
                    ok = fabs(s - (i == j)) < 1e-12;
                }
            if (ok) hm.pinv[p] = q;
        }
    for (int p = 0; p < nst; ++p)
        if (hm.pinv[p] < 0) return hm;
    std::vector<std::vector<std::pair<int, double>>> rows((size_t)nst * PS);
    for (int p = 0; p < nst; ++p) {
        const double *P = a.sml + (size_t)p * n * n, *Sm = a.sms + (size_t)p * m * m;
        for (int x = 0; x < n; ++x)
            for (int y = 0; y <= x; ++y) {
                std::vector<double> c(T, 0.0);
                for (int u = 0; u < n; ++u)
                    for (int v = 0; v < n; ++v) c[sx(u, v)] += P[x * n + u] * P[y * n + v];
                for (int s2 = 0; s2 < T; ++s2)
                    if (c[s2] != 0.0) rows[(size_t)p * PS + sx(x, y)].push_back({s2, c[s2]});
            }
        rows[(size_t)p * PS + T].push_back({T, 1.0});
        for (int r = 0; r < m; ++r)
            for (int u = 0; u < m; ++u)
                if (Sm[u * m + r] != 0.0) rows[(size_t)p * PS + T + 1 + r].push_back({T + 1 + u, Sm[u * m + r]});
    }
    for (auto &r : rows) hm.maxnz = (int)r.size() > hm.maxnz ? (int)r.size() : hm.maxnz;
    hm.cnt.resize(rows.size());
    hm.src.assign(rows.size() * hm.maxnz, 0);
    hm.coef.assign(rows.size() * hm.maxnz, 0.0);
    for (size_t e = 0; e < rows.size(); ++e) {
        hm.cnt[e] = (int)rows[e].size();
        for (size_t i = 0; i < rows[e].size(); ++i) {
            hm.src[e * hm.maxnz + i] = rows[e][i].first;
            hm.coef[e * hm.maxnz + i] = rows[e][i].second;
        }
    }
    hm.ok = true;
    return hm;
}

struct RowOutH {
    double *r;
    void put(int f, CD v) { r[f] = v.v; }
    void add(int f, CD v) { r[f] += v.v; }
};
// the fused pass's ket output: the H and S values of one field together
struct RowOutHS {
    double *rh, *rs;
    void put(int f, CD vh, CD vs) {
        rh[f] = vh.v;
        rs[f] = vs.v;
    }
    void add(int f, CD vh, CD vs) {
        rh[f] += vh.v;
        rs[f] += vs.v;
    }
};

template <int N> int outprod_sym(const Args &a, const double *x, int LCe, int LCs, double *f, double *g, double *H,
                                 double *S) {
    const int K = a.K, nst = a.nst;
    constexpr int PS = Part<N>::size;
    if (PS > 32) return -2;
    const size_t siv = (size_t)K * (tri(N) + 3 * N);
    const double *iv = x, *C = x + siv;
    HostMap hm = build_map<N>(a);
    if (!hm.ok) return -3;
    Consts<N> cs = consts<N>(a.mass, a.ncv, a.efs);
    std::vector<double> bra((size_t)BraLayout<N>::size * K), ket((size_t)KetLayout<N>::size * K * nst);
    for (int k = 0; k < K; ++k) prep_bra_one<N>(iv, K, cs, bra.data(), k);
    for (int id = 0; id < K * nst; ++id)
        prep_ket_one<N>(iv, C, nst, cs, a.sml, a.sms, a.scvv, ket.data(), id, hm.pinv.data());
    int flags = 0;
    for (int kb = 0; kb * 32 < K; ++kb)
        for (int lc = 0; lc * LCe <= kb * 32 + 31 && lc * LCe < K; ++lc)
            for (int lane = 0; lane < 32; ++lane) {
                int k, l0, lend, bad = 0;
                if (!energy_lane_range(kb, lc, lane, LCe, K, k, l0, lend)) continue;
                flags |= energy_lane<N, CD>(HostBra{bra.data() + k, (size_t)K}, HostKetBase{ket.data()}, k, l0,
                                            lend, K, nst, cs, H, S, nullptr, nullptr, bad);
            }
    std::vector<double> rh(K), rs(K);
    double cHc = 0.0, cSc = 0.0;
    for (int i = 0; i < K; ++i) {
        double hh = 0.0, ss = 0.0;
        for (int j = 0; j < K; ++j) {
            hh += H[(size_t)i * K + j] * C[j];
            ss += S[(size_t)i * K + j] * C[j];
        }
        rh[i] = hh;
        rs[i] = ss;
        cHc += C[i] * hh;
        cSc += C[i] * ss;
    }
    const double E = cHc / cSc, norm = 1.0 / cSc;
    *f = E;
    for (int i = 0; i < K; ++i) g[siv + i] = 2.0 * norm * (rh[i] - E * rs[i]);
    // symmetric tiles
    std::vector<int> tstart;
    std::vector<std::pair<int, int>> tiles;
    for (int kb = 0; kb * 32 < K; ++kb) {
        tstart.push_back((int)tiles.size());
        const int last = kb * 32 + 31 < K - 1 ? kb * 32 + 31 : K - 1;
        for (int lc = 0; lc <= last / LCs; ++lc) tiles.push_back({kb, lc});
    }
    tstart.push_back((int)tiles.size());
    const int nt = (int)tiles.size();
    std::vector<double> pb((size_t)nt * PS * 32, 0.0), pk((size_t)nt * LCs * PS, 0.0);
    KetMap km{hm.cnt.data(), hm.src.data(), hm.coef.data(), hm.maxnz};
    for (int t = 0; t < nt; ++t) {
        const int kb = tiles[t].first, l0 = tiles[t].second * LCs, l1 = std::min(l0 + LCs, K);
        std::vector<RegAcc<N, CD>> accs(32);
        for (auto &ac : accs) ac.zero();
        for (int l = l0; l < l1; ++l) {
            double accl[32] = {0.0};
            for (int P = 0; P < nst; ++P) {
                const double *krp = ket.data() + ((size_t)l * nst + P) * KetLayout<N>::size;
                double rows[32][33];
                for (int lane = 0; lane < 32; ++lane) {
                    const int k = kb * 32 + lane;
                    for (int ff = 0; ff < PS; ++ff) rows[lane][ff] = 0.0;
                    if (k < K && l <= k) {
                        const double wk = l < k ? 2.0 * C[k] * krp[KetLayout<N>::winv] : 0.0;
                        RowOutH ro{rows[lane]};
                        if (!term_sym<N, CD>(HostBra{bra.data() + k, (size_t)K}, HostKet{krp}, cs, CD(E),
                                             CD(krp[KetLayout<N>::wC]), CD(wk), accs[lane], ro))
                            flags |= 1;
                    }
                }
                double red[32];
                for (int j = 0; j < 32; ++j) {
                    double v = 0.0;
                    if (j < PS)
                        for (int r = 0; r < 32; ++r) v += rows[r][j];
                    red[j] = v;
                }
                for (int j = 0; j < PS; ++j) accl[j] += ket_map_apply(km, P, j, PS, red);
            }
            for (int j = 0; j < PS; ++j) pk[((size_t)t * LCs + (l - l0)) * PS + j] = accl[j];
        }
        for (int lane = 0; lane < 32; ++lane) {
            if (kb * 32 + lane >= K) continue;
            for (int tt = 0; tt < tri(N); ++tt) pb[((size_t)t * PS + tt) * 32 + lane] = accs[lane].g(tt).v;
            pb[((size_t)t * PS + tri(N)) * 32 + lane] = accs[lane].d().v;
            for (int tt = 0; tt < 3 * N; ++tt) pb[((size_t)t * PS + tri(N) + 1 + tt) * 32 + lane] = accs[lane].s(tt).v;
        }
    }
    std::vector<double> out((size_t)PS * K, 0.0);
    const int nkb = (K + 31) / 32;
    for (int ff = 0; ff < PS; ++ff)
        for (int m = 0; m < K; ++m) {
            const int kb = m / 32, lane = m % 32;
            double s = 0.0;
            for (int t = tstart[kb]; t < tstart[kb + 1]; ++t) s += pb[((size_t)t * PS + ff) * 32 + lane];
            const int lc = m / LCs, ll = m % LCs;
            int kb0 = lc * LCs - 31;
            kb0 = kb0 > 0 ? (kb0 + 31) / 32 : 0;
            for (int q = kb0; q < nkb; ++q) s += pk[((size_t)(tstart[q] + lc) * LCs + ll) * PS + ff];
            out[(size_t)ff * K + m] = s;
        }
    for (int k = 0; k < K; ++k)
        if (!grad_reduce_one<N>(out.data(), 1, K, bra.data(), norm * C[k], g, k)) flags |= 2;
    return flags;
}

// Host mirror of the fused pass (fsym_kernel + fsym_sum_kernel): one pass over
// unordered pairs writes H and S and keeps the H and S gradients apart; after
// finalize computes E they are combined as g_H - E g_S.
template <int N> int outprod_fused(const Args &a, const double *x, int LCs, double *f, double *g, double *H,
                                   double *S) {
    const int K = a.K, nst = a.nst;
    constexpr int PS = Part<N>::size;
    if (PS > 32) return -2;
    const size_t siv = (size_t)K * (tri(N) + 3 * N);
    const double *iv = x, *C = x + siv;
    HostMap hm = build_map<N>(a);
    if (!hm.ok) return -3;
    Consts<N> cs = consts<N>(a.mass, a.ncv, a.efs);
    std::vector<double> bra((size_t)BraLayout<N>::size * K), ket((size_t)KetLayout<N>::size * K * nst);
    for (int k = 0; k < K; ++k) prep_bra_one<N>(iv, K, cs, bra.data(), k);
    for (int id = 0; id < K * nst; ++id)
        prep_ket_one<N>(iv, C, nst, cs, a.sml, a.sms, a.scvv, ket.data(), id, hm.pinv.data());
    int flags = 0;
    std::vector<int> tstart;
    std::vector<std::pair<int, int>> tiles;
    for (int kb = 0; kb * 32 < K; ++kb) {
        tstart.push_back((int)tiles.size());
        const int last = kb * 32 + 31 < K - 1 ? kb * 32 + 31 : K - 1;
        for (int lc = 0; lc <= last / LCs; ++lc) tiles.push_back({kb, lc});
    }
    tstart.push_back((int)tiles.size());
    const int nt = (int)tiles.size();
    std::vector<double> pb((size_t)nt * 2 * PS * 32, 0.0), pk((size_t)nt * LCs * 2 * PS, 0.0);
    KetMap km{hm.cnt.data(), hm.src.data(), hm.coef.data(), hm.maxnz};
    for (int t = 0; t < nt; ++t) {
        const int kb = tiles[t].first, l0 = tiles[t].second * LCs, l1 = std::min(l0 + LCs, K);
        std::vector<RegAcc<N, CD>> accH(32), accS(32);
        for (int lane = 0; lane < 32; ++lane) {
            accH[lane].zero();
            accS[lane].zero();
        }
        for (int l = l0; l < l1; ++l) {
            double aH[32] = {0.0}, aS[32] = {0.0};
            double hsum[32] = {0.0}, ssum[32] = {0.0};
            for (int P = 0; P < nst; ++P) {
                const double *krp = ket.data() + ((size_t)l * nst + P) * KetLayout<N>::size;
                double rowsH[32][33], rowsS[32][33];
                for (int lane = 0; lane < 32; ++lane) {
                    const int k = kb * 32 + lane;
                    for (int ff = 0; ff < PS; ++ff) rowsH[lane][ff] = rowsS[lane][ff] = 0.0;
                    if (k < K && l <= k) {
                        const double wk = l < k ? 2.0 * C[k] * krp[KetLayout<N>::winv] : 0.0;
                        RowOutHS ro{rowsH[lane], rowsS[lane]};
                        CD h, ov;
                        if (!term_fused<N, CD>(HostBra{bra.data() + k, (size_t)K}, HostKet{krp}, cs,
                                               CD(krp[KetLayout<N>::wC]), CD(wk), accH[lane], accS[lane], ro, h,
                                               ov))
                            flags |= 1;
                        const double w = krp[KetLayout<N>::w];
                        hsum[lane] += w * h.v;
                        ssum[lane] += w * ov.v;
                    }
                }
                // the kernel adds lane pairs (2i, 2i+1) by shuffle, then the 16 rows
                for (int which = 0; which < 2; ++which) {
                    double red[32];
                    for (int j = 0; j < 32; ++j) {
                        double v = 0.0;
                        if (j < PS)
                            for (int r = 0; r < 16; ++r)
                                v += which ? rowsS[2 * r][j] + rowsS[2 * r + 1][j]
                                           : rowsH[2 * r][j] + rowsH[2 * r + 1][j];
                        red[j] = v;
                    }
                    for (int j = 0; j < PS; ++j) (which ? aS : aH)[j] += ket_map_apply(km, P, j, PS, red);
                }
            }
            for (int lane = 0; lane < 32; ++lane) {
                const int k = kb * 32 + lane;
                if (k < K && l <= k) {
                    if (!std::isfinite(hsum[lane]) || !std::isfinite(ssum[lane])) flags |= 2;
                    H[(size_t)k * K + l] = H[(size_t)l * K + k] = hsum[lane];
                    S[(size_t)k * K + l] = S[(size_t)l * K + k] = ssum[lane];
                }
            }
            for (int j = 0; j < PS; ++j) {
                pk[(((size_t)t * LCs + (l - l0)) * 2 + 0) * PS + j] = aH[j];
                pk[(((size_t)t * LCs + (l - l0)) * 2 + 1) * PS + j] = aS[j];
            }
        }
        for (int lane = 0; lane < 32; ++lane) {
            if (kb * 32 + lane >= K) continue;
            for (int which = 0; which < 2; ++which) {
                RegAcc<N, CD> &ac = which ? accS[lane] : accH[lane];
                const size_t base = ((size_t)t * 2 + which) * PS;
                for (int tt = 0; tt < tri(N); ++tt) pb[(base + tt) * 32 + lane] = ac.g(tt).v;
                pb[(base + tri(N)) * 32 + lane] = ac.d().v;
                for (int tt = 0; tt < 3 * N; ++tt) pb[(base + tri(N) + 1 + tt) * 32 + lane] = ac.s(tt).v;
            }
        }
    }
    // rows + finalize
    std::vector<double> rh(K), rs(K);
    double cHc = 0.0, cSc = 0.0;
    for (int i = 0; i < K; ++i) {
        double hh = 0.0, ss = 0.0;
        for (int j = 0; j < K; ++j) {
            hh += H[(size_t)i * K + j] * C[j];
            ss += S[(size_t)i * K + j] * C[j];
        }
        rh[i] = hh;
        rs[i] = ss;
        cHc += C[i] * hh;
        cSc += C[i] * ss;
    }
    const double E = cHc / cSc, norm = 1.0 / cSc;
    *f = E;
    for (int i = 0; i < K; ++i) g[siv + i] = 2.0 * norm * (rh[i] - E * rs[i]);
    std::vector<double> out((size_t)PS * K, 0.0);
    const int nkb = (K + 31) / 32;
    for (int ff = 0; ff < PS; ++ff)
        for (int m = 0; m < K; ++m) {
            const int kb = m / 32, lane = m % 32;
            // the kernel's order: 8 segments (every 8th tile), combined in order
            double segH[8] = {0.0}, segS[8] = {0.0};
            for (int q = 0; q < 8; ++q)
                for (int t = tstart[kb] + q; t < tstart[kb + 1]; t += 8) {
                    segH[q] += pb[(((size_t)t * 2 + 0) * PS + ff) * 32 + lane];
                    segS[q] += pb[(((size_t)t * 2 + 1) * PS + ff) * 32 + lane];
                }
            double sH = segH[0], sS = segS[0];
            for (int q = 1; q < 8; ++q) {
                sH += segH[q];
                sS += segS[q];
            }
            const int lc = m / LCs, ll = m % LCs;
            int kb0 = lc * LCs - 31;
            kb0 = kb0 > 0 ? (kb0 + 31) / 32 : 0;
            for (int q = kb0; q < nkb; ++q) {
                const size_t base = ((size_t)(tstart[q] + lc) * LCs + ll) * 2;
                sH += pk[(base + 0) * PS + ff];
                sS += pk[(base + 1) * PS + ff];
            }
            out[(size_t)ff * K + m] = sH - E * sS;
        }
    for (int k = 0; k < K; ++k)
        if (!grad_reduce_one<N>(out.data(), 1, K, bra.data(), norm * C[k], g, k)) flags |= 2;
    return flags;
}

// Host mirror of rrms_kernel (per term) and of dipole_kernel + dipole_sum_kernel
// (energy tiles in the device list order, per-lane sums over (Pe, l, P), the
// warp's butterfly sum, tile partials summed by 256 strided threads and a tree).
template <int N> int rrms_terms(const Args &a, const double *iv, int nterms, const int *terms, double *out) {
    using KL = KetLayout<N>;
    Consts<N> cs = consts<N>(a.mass, a.ncv, a.efs);
    std::vector<double> bra, ket;
    prep<N>(a, iv, nullptr, bra, ket, cs);
    int flags = 0;
    for (int t = 0; t < nterms; ++t) {
        const int *q = terms + 5 * t;
        const int stfe = q[0] - 1, stf = q[1] - 1, ii = q[2] - 1, jj = q[3] - 1, n1 = q[4] - 1;
        CD T[3 * N], ov;
        if (!term_dipole<N, CD>(HostKet{ket.data() + ((size_t)ii * a.nst + stfe) * KL::size},
                                HostKet{ket.data() + ((size_t)jj * a.nst + stf) * KL::size}, cs, T, ov))
            flags |= 1;
        out[2 * t] = ov.v;
        out[2 * t + 1] = T[n1].v * ov.v;
    }
    return flags;
}

template <int N> int dipole(const Args &a, const double *iv, const double *C, int LC, double *comps, double *dip) {
    using KL = KetLayout<N>;
    constexpr int NM = 3 * N + 1;
    const int K = a.K, nst = a.nst;
    Consts<N> cs = consts<N>(a.mass, a.ncv, a.efs);
    std::vector<double> bra, ket;
    prep<N>(a, iv, C, bra, ket, cs);
    int flags = 0;
    std::vector<double> part;
    for (int kb = 0; kb * 32 < K; ++kb)
        for (int lc = 0; lc * LC <= kb * 32 + 31 && lc * LC < K; ++lc) {
            double acc[32][NM] = {};
            for (int lane = 0; lane < 32; ++lane) {
                int k, l0, lend;
                if (!energy_lane_range(kb, lc, lane, LC, K, k, l0, lend)) continue;
                for (int Pe = 0; Pe < nst; ++Pe) {
                    const double *kbr = ket.data() + ((size_t)k * nst + Pe) * KL::size;
                    const double wek = kbr[KL::w] * C[k];
                    for (int l = l0; l < lend; ++l) {
                        const double wl = (l == k ? 1.0 : 2.0) * wek * C[l];
                        for (int P = 0; P < nst; ++P) {
                            const double *kr = ket.data() + ((size_t)l * nst + P) * KL::size;
                            CD T[3 * N], ov;
                            if (!term_dipole<N, CD>(HostKet{kbr}, HostKet{kr}, cs, T, ov)) flags |= 1;
                            const double wo = wl * kr[KL::w] * ov.v;
                            acc[lane][0] += wo;
                            for (int m = 0; m < 3 * N; ++m) acc[lane][1 + m] += wo * T[m].v;
                        }
                    }
                }
            }
            for (int m = 0; m < NM; ++m) {  // butterfly: xor 16, 8, 4, 2, 1
                double v[32];
                for (int lane = 0; lane < 32; ++lane) v[lane] = acc[lane][m];
                for (int o = 16; o > 0; o >>= 1) {
                    double w[32];
                    for (int lane = 0; lane < 32; ++lane) w[lane] = v[lane] + v[lane ^ o];
                    for (int lane = 0; lane < 32; ++lane) v[lane] = w[lane];
                }
                part.push_back(v[0]);
            }
        }
    const int ntiles = (int)(part.size() / NM);
    double tot[NM];
    for (int m = 0; m < NM; ++m) {
        double red[256];
        for (int j = 0; j < 256; ++j) {
            double s = 0.0;
            for (int t = j; t < ntiles; t += 256) s += part[(size_t)t * NM + m];
            red[j] = s;
        }
        for (int w = 128; w > 0; w >>= 1)
            for (int j = 0; j < w; ++j) red[j] += red[j + w];
        tot[m] = red[0];
    }
    for (int m = 0; m < 3 * N; ++m) comps[m] = tot[0] != 0.0 ? tot[1 + m] / tot[0] : 0.0;
    for (int c = 0; c < 3; ++c) {
        double d = 0.0;
        for (int i = 0; i < N; ++i) d += cs.q[i] * comps[3 * i + c];
        dip[c] = d;
    }
    return flags;
}

// Host mirror of one rank's share of a sharded evaluation (necg_shard_pairs and
// the per-basis sums of necg_shard_grad): the fused tiles [t0, t1) only, with
// H and S zero outside them; returns this shard's rows (H C, S C) and its
// per-basis sums of the H and of the S gradient partials, kept apart (the
// caller combines them once E is known from the summed rows).
template <int N> int shard_pairs(const Args &a, const double *x, int LCs, int t0, int t1, double *rows,
                                 double *sumH, double *sumS, int *ntiles_out) {
    const int K = a.K, nst = a.nst;
    constexpr int PS = Part<N>::size;
    if (PS > 32) return -2;
    const size_t siv = (size_t)K * (tri(N) + 3 * N);
    const double *iv = x, *C = x + siv;
    HostMap hm = build_map<N>(a);
    if (!hm.ok) return -3;
    Consts<N> cs = consts<N>(a.mass, a.ncv, a.efs);
    std::vector<double> bra((size_t)BraLayout<N>::size * K), ket((size_t)KetLayout<N>::size * K * nst);
    for (int k = 0; k < K; ++k) prep_bra_one<N>(iv, K, cs, bra.data(), k);
    for (int id = 0; id < K * nst; ++id)
        prep_ket_one<N>(iv, C, nst, cs, a.sml, a.sms, a.scvv, ket.data(), id, hm.pinv.data());
    std::vector<int> tstart;
    std::vector<std::pair<int, int>> tiles;
    for (int kb = 0; kb * 32 < K; ++kb) {
        tstart.push_back((int)tiles.size());
        const int last = kb * 32 + 31 < K - 1 ? kb * 32 + 31 : K - 1;
        for (int lc = 0; lc <= last / LCs; ++lc) tiles.push_back({kb, lc});
    }
    tstart.push_back((int)tiles.size());
    const int nt = (int)tiles.size();
    *ntiles_out = nt;
    if (t0 < 0 || t1 > nt || t1 < t0) return -4;
    std::vector<double> H((size_t)K * K, 0.0), S((size_t)K * K, 0.0);
    std::vector<double> pb((size_t)nt * 2 * PS * 32, 0.0), pk((size_t)nt * LCs * 2 * PS, 0.0);
    KetMap km{hm.cnt.data(), hm.src.data(), hm.coef.data(), hm.maxnz};
    int flags = 0;
    for (int t = t0; t < t1; ++t) {
        const int kb = tiles[t].first, l0 = tiles[t].second * LCs, l1 = std::min(l0 + LCs, K);
        std::vector<RegAcc<N, CD>> accH(32), accS(32);
        for (int lane = 0; lane < 32; ++lane) {
            accH[lane].zero();
            accS[lane].zero();
        }
        for (int l = l0; l < l1; ++l) {
            double aH[32] = {0.0}, aS[32] = {0.0};
            double hsum[32] = {0.0}, ssum[32] = {0.0};
            for (int P = 0; P < nst; ++P) {
                const double *krp = ket.data() + ((size_t)l * nst + P) * KetLayout<N>::size;
                double rowsH[32][33], rowsS[32][33];
                for (int lane = 0; lane < 32; ++lane) {
                    const int k = kb * 32 + lane;
                    for (int ff = 0; ff < PS; ++ff) rowsH[lane][ff] = rowsS[lane][ff] = 0.0;
                    if (k < K && l <= k) {
                        const double wk = l < k ? 2.0 * C[k] * krp[KetLayout<N>::winv] : 0.0;
                        RowOutHS ro{rowsH[lane], rowsS[lane]};
                        CD h, ov;
                        if (!term_fused<N, CD>(HostBra{bra.data() + k, (size_t)K}, HostKet{krp}, cs,
                                               CD(krp[KetLayout<N>::wC]), CD(wk), accH[lane], accS[lane], ro, h,
                                               ov))
                            flags |= 1;
                        hsum[lane] += krp[KetLayout<N>::w] * h.v;
                        ssum[lane] += krp[KetLayout<N>::w] * ov.v;
                    }
                }
                for (int which = 0; which < 2; ++which) {
                    double red[32];
                    for (int j = 0; j < 32; ++j) {
                        double v = 0.0;
                        if (j < PS)
                            for (int r = 0; r < 16; ++r)
                                v += which ? rowsS[2 * r][j] + rowsS[2 * r + 1][j]
                                           : rowsH[2 * r][j] + rowsH[2 * r + 1][j];
                        red[j] = v;
                    }
                    for (int j = 0; j < PS; ++j) (which ? aS : aH)[j] += ket_map_apply(km, P, j, PS, red);
                }
            }
            for (int lane = 0; lane < 32; ++lane) {
                const int k = kb * 32 + lane;
                if (k < K && l <= k) {
                    H[(size_t)k * K + l] = H[(size_t)l * K + k] = hsum[lane];
                    S[(size_t)k * K + l] = S[(size_t)l * K + k] = ssum[lane];
                }
            }
            for (int j = 0; j < PS; ++j) {
                pk[(((size_t)t * LCs + (l - l0)) * 2 + 0) * PS + j] = aH[j];
                pk[(((size_t)t * LCs + (l - l0)) * 2 + 1) * PS + j] = aS[j];
            }
        }
        for (int lane = 0; lane < 32; ++lane) {
            if (kb * 32 + lane >= K) continue;
            for (int which = 0; which < 2; ++which) {
                RegAcc<N, CD> &ac = which ? accS[lane] : accH[lane];
                const size_t base = ((size_t)t * 2 + which) * PS;
                for (int tt = 0; tt < tri(N); ++tt) pb[(base + tt) * 32 + lane] = ac.g(tt).v;
                pb[(base + tri(N)) * 32 + lane] = ac.d().v;
                for (int tt = 0; tt < 3 * N; ++tt) pb[(base + tri(N) + 1 + tt) * 32 + lane] = ac.s(tt).v;
            }
        }
    }
    for (int i = 0; i < K; ++i) {
        double hh = 0.0, ss = 0.0;
        for (int j = 0; j < K; ++j) {
            hh += H[(size_t)i * K + j] * C[j];
            ss += S[(size_t)i * K + j] * C[j];
        }
        rows[i] = hh;
        rows[K + i] = ss;
    }
    const int nkb = (K + 31) / 32;
    for (int ff = 0; ff < PS; ++ff)
        for (int m = 0; m < K; ++m) {
            const int kb = m / 32, lane = m % 32;
            const int ta = std::max(tstart[kb], t0), tb = std::min(tstart[kb + 1], t1);
            double segH[8] = {0.0}, segS[8] = {0.0};
            for (int q = 0; q < 8; ++q)
                for (int t = ta + q; t < tb; t += 8) {
                    segH[q] += pb[(((size_t)t * 2 + 0) * PS + ff) * 32 + lane];
                    segS[q] += pb[(((size_t)t * 2 + 1) * PS + ff) * 32 + lane];
                }
            double sH = segH[0], sS = segS[0];
            for (int q = 1; q < 8; ++q) {
                sH += segH[q];
                sS += segS[q];
            }
            const int lc = m / LCs, ll = m % LCs;
            int kb0 = lc * LCs - 31;
            kb0 = kb0 > 0 ? (kb0 + 31) / 32 : 0;
            for (int q = kb0; q < nkb; ++q) {
                const int t = tstart[q] + lc;
                if (t < t0 || t >= t1) continue;
                const size_t base = ((size_t)t * LCs + ll) * 2;
                sH += pk[(base + 0) * PS + ff];
                sS += pk[(base + 1) * PS + ff];
            }
            sumH[(size_t)ff * K + m] = sH;
            sumS[(size_t)ff * K + m] = sS;
        }
    return flags;
}

// GRADA from summed per-basis sums (necg_shard_finish): g[block k] from
// sums[f * K + k] scaled by norm C_k.
template <int N> int shard_finish(const Args &a, const double *x, const double *sums, double norm, double *g) {
    const int K = a.K;
    const size_t siv = (size_t)K * (tri(N) + 3 * N);
    Consts<N> cs = consts<N>(a.mass, a.ncv, a.efs);
    std::vector<double> bra((size_t)BraLayout<N>::size * K);
    for (int k = 0; k < K; ++k) prep_bra_one<N>(x, K, cs, bra.data(), k);
    int flags = 0;
    for (int k = 0; k < K; ++k)
        if (!grad_reduce_one<N>(sums, 1, K, bra.data(), norm * x[siv + k], g, k)) flags |= 2;
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

extern "C" int emu_outprod_sym(int n, int nst, int K, double efs, const double *mass, const double *ncv,
                               const double *scvv, const double *sml, const double *sms, const double *x,
                               int lc_e, int lc_s, double *f, double *g, double *H, double *S) {
    Args a{nst, K, efs, mass, ncv, scvv, sml, sms};
    EMU_DISPATCH(n, (outprod_sym<N>(a, x, lc_e, lc_s, f, g, H, S)));
}

extern "C" int emu_outprod_fused(int n, int nst, int K, double efs, const double *mass, const double *ncv,
                                 const double *scvv, const double *sml, const double *sms, const double *x,
                                 int lc_s, double *f, double *g, double *H, double *S) {
    Args a{nst, K, efs, mass, ncv, scvv, sml, sms};
    EMU_DISPATCH(n, (outprod_fused<N>(a, x, lc_s, f, g, H, S)));
}

extern "C" int emu_rrms(int n, int nst, int K, double efs, const double *mass, const double *ncv,
                        const double *scvv, const double *sml, const double *sms, const double *iv, int nterms,
                        const int *terms, double *out) {
    Args a{nst, K, efs, mass, ncv, scvv, sml, sms};
    EMU_DISPATCH(n, (rrms_terms<N>(a, iv, nterms, terms, out)));
}

extern "C" int emu_dipole(int n, int nst, int K, double efs, const double *mass, const double *ncv,
                          const double *scvv, const double *sml, const double *sms, const double *iv,
                          const double *C, int lc, double *comps, double *dip) {
    Args a{nst, K, efs, mass, ncv, scvv, sml, sms};
    EMU_DISPATCH(n, (dipole<N>(a, iv, C, lc, comps, dip)));
}

extern "C" int emu_shard_pairs(int n, int nst, int K, double efs, const double *mass, const double *ncv,
                               const double *scvv, const double *sml, const double *sms, const double *x,
                               int lc_s, int t0, int t1, double *rows, double *sumH, double *sumS,
                               int *ntiles) {
    Args a{nst, K, efs, mass, ncv, scvv, sml, sms};
    EMU_DISPATCH(n, (shard_pairs<N>(a, x, lc_s, t0, t1, rows, sumH, sumS, ntiles)));
}

extern "C" int emu_shard_finish(int n, int nst, int K, double efs, const double *mass, const double *ncv,
                                const double *scvv, const double *sml, const double *sms, const double *x,
                                const double *sums, double norm, double *g) {
    Args a{nst, K, efs, mass, ncv, scvv, sml, sms};
    EMU_DISPATCH(n, (shard_finish<N>(a, x, sums, norm, g)));
}

extern "C" int emu_elements(int n, int nst, int K, double efs, const double *mass, const double *ncv,
                            const double *scvv, const double *sml, const double *sms, const double *iv,
                            int nterms, const int *terms, double *mat, double *tg, double *tgs) {
    Args a{nst, K, efs, mass, ncv, scvv, sml, sms};
    EMU_DISPATCH(n, (elements<N>(a, iv, nterms, terms, mat, tg, tgs)));
}
