// necg_hostscalar.cuh -- a value-carrying FP64 scalar that also counts the
// operations applied to it, and host accessors for bra/ket records.  Used to
// instantiate the term templates of necg_math.cuh on the host: by the FLOP
// counter (necg_count.cu) and by the test emulator of the kernels.
#pragma once
#include <math.h>
#include <stddef.h>

namespace necg {

struct CountCtx {
    long long flops = 0, special = 0;
};
inline CountCtx &count_ctx() {
    static thread_local CountCtx c;
    return c;
}

struct CD {
    double v;
    CD() : v(0.0) {}
    CD(double x) : v(x) {}
    CD &operator+=(const CD &o) { ++count_ctx().flops; v += o.v; return *this; }
    CD &operator-=(const CD &o) { ++count_ctx().flops; v -= o.v; return *this; }
    CD &operator*=(const CD &o) { ++count_ctx().flops; v *= o.v; return *this; }
};
inline CD operator+(CD a, CD b) { ++count_ctx().flops; return CD(a.v + b.v); }
inline CD operator-(CD a, CD b) { ++count_ctx().flops; return CD(a.v - b.v); }
inline CD operator*(CD a, CD b) { ++count_ctx().flops; return CD(a.v * b.v); }
inline CD operator/(CD a, CD b) { ++count_ctx().special; return CD(a.v / b.v); }
inline CD operator+(double a, CD b) { return CD(a) + b; }
inline CD operator+(CD a, double b) { return a + CD(b); }
inline CD operator-(double a, CD b) { return CD(a) - b; }
inline CD operator-(CD a, double b) { return a - CD(b); }
inline CD operator*(double a, CD b) { return CD(a) * b; }
inline CD operator*(CD a, double b) { return a * CD(b); }
inline CD operator-(CD a) { return CD(-a.v); }
inline bool operator>(CD a, double b) { return a.v > b; }
inline bool operator<=(CD a, double b) { return a.v <= b; }
inline bool operator<=(CD a, CD b) { return a.v <= b.v; }
inline CD sqrt(CD a) { ++count_ctx().special; return CD(::sqrt(a.v)); }
inline CD rsqrt(CD a) { ++count_ctx().special; return CD(1.0 / ::sqrt(a.v)); }
inline CD rsq(CD a) { return rsqrt(a); }
inline CD rcp(CD a) { return CD(1.0) / a; }
inline CD exp(CD a) { ++count_ctx().special; return CD(::exp(a.v)); }
inline double val(CD x) { return x.v; }

// bra record field f of basis k in a structure-of-arrays buffer
struct HostBra {
    const double *p;  // bra + k
    size_t K;
    CD operator()(int f) const { return CD(p[(size_t)f * K]); }
};
struct HostKet {
    const double *p;
    CD operator[](int i) const { return CD(p[i]); }
};
struct HostKetBase {
    const double *p;
    HostKet at(size_t off) const { return HostKet{p + off}; }
};

}  // namespace necg
