// cosmology.cpp -- host binary64 scalars of the KDK step (include/hyowon_cosmology.h).
//
// Written from the mathematics of flat matter + Lambda:
//   E(a) = sqrt(Om a^-3 + OL), H = 100 E  (km/s/(Mpc/h));
//   D(a1,a2) = int da/(a^3 H), K(a1,a2) = int da/(a^2 H)
//     evaluated in u = ln(a/a1) as int du/(a (aH)) and int du/(aH);
//   steps uniform in ln a, a_k = a0 (1 + expm1(k dlna)), exact final stop,
//   midpoint a_half = correctly rounded sqrt(a_begin a_end);
//   D1 ~ E(a) int_0^a da'/(a'E)^3 (the growing mode), f1 = dlnD1/dlna.
// The quadrature is a composite Gauss-Legendre rule whose nodes are computed
// here by Newton iteration on Legendre polynomials; it refines by cell
// doubling until the 8/16-point gap and the change under doubling are both
// within one binary64 spacing of the result.
#include "hyowon_cosmology.h"

#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>

namespace {

constexpr int kOk = 0;
constexpr int kInvalid = 1;
constexpr int kOverflow = 3;

template <int Order>
struct GaussLegendre {
    // Positive half of the symmetric nodes and their weights on [-1, 1].
    std::array<double, Order / 2> x{};
    std::array<double, Order / 2> w{};
    GaussLegendre() {
        const long double pi = 3.141592653589793238462643383279502884L;
        for (int i = 0; i < Order / 2; ++i) {
            long double z = std::cos(pi * (i + 0.75L) / (Order + 0.5L));
            long double dp = 0.0L;
            for (int it = 0; it < 100; ++it) {
                long double p0 = 1.0L, p1 = z;
                for (int k = 2; k <= Order; ++k) {
                    const long double p2 = ((2.0L * k - 1.0L) * z * p1 - (k - 1.0L) * p0) / k;
                    p0 = p1;
                    p1 = p2;
                }
                dp = Order * (z * p1 - p0) / (z * z - 1.0L);
                const long double dz = p1 / dp;
                z -= dz;
                if (std::fabs(dz) < 1e-19L) break;
            }
            x[i] = static_cast<double>(z);
            w[i] = static_cast<double>(2.0L / ((1.0L - z * z) * dp * dp));
        }
    }
};

const GaussLegendre<16>& gl16() {
    static const GaussLegendre<16> g;
    return g;
}
const GaussLegendre<8>& gl8() {
    static const GaussLegendre<8> g;
    return g;
}

struct Cosmo {
    double om, ol;
    double sqrt_m, sqrt_l;
    Cosmo(double m, double l) : om(m), ol(l), sqrt_m(std::sqrt(m)), sqrt_l(std::sqrt(l)) {}
    double E(double a) const {
        const double sa = std::sqrt(a);
        const double matter = sqrt_m / (a * sa);
        return std::hypot(matter, sqrt_l);
    }
    double H(double a) const { return 100.0 * E(a); }
};

bool valid_cosmology(double om, double ol) {
    return std::isfinite(om) && std::isfinite(ol) && om > 0.0 && om <= 1.0 && ol >= 0.0
        && std::fabs(om + ol - 1.0) <= 4.0 * std::numeric_limits<double>::epsilon();
}

void compensated(long double term, long double& sum, long double& comp) {
    const long double t = sum + term;
    if (std::fabs(sum) >= std::fabs(term)) comp += (sum - t) + term;
    else comp += (term - t) + sum;
    sum = t;
}

double spacing(double v) {
    const double up = std::nextafter(v, std::numeric_limits<double>::infinity());
    const double dn = std::nextafter(v, -std::numeric_limits<double>::infinity());
    return std::fmax(up - v, v - dn);
}

template <typename F>
void composite(const F& f, double lo, double hi, std::size_t cells, long double& i8,
               long double& i16) {
    const double width = hi - lo;
    const double cw = width / static_cast<double>(cells);
    const double hw = 0.5 * cw;
    long double s8 = 0, c8 = 0, s16 = 0, c16 = 0;
    for (std::size_t c = 0; c < cells; ++c) {
        const double mid = lo + (static_cast<double>(c) + 0.5) * cw;
        long double l8 = 0, lc8 = 0, l16 = 0, lc16 = 0;
        for (int i = 0; i < 4; ++i) {
            const double o = hw * gl8().x[i];
            compensated(static_cast<long double>(gl8().w[i])
                            * (static_cast<long double>(f(mid - o)) + f(mid + o)),
                        l8, lc8);
        }
        for (int i = 0; i < 8; ++i) {
            const double o = hw * gl16().x[i];
            compensated(static_cast<long double>(gl16().w[i])
                            * (static_cast<long double>(f(mid - o)) + f(mid + o)),
                        l16, lc16);
        }
        compensated(static_cast<long double>(hw) * (l8 + lc8), s8, c8);
        compensated(static_cast<long double>(hw) * (l16 + lc16), s16, c16);
    }
    i8 = s8 + c8;
    i16 = s16 + c16;
}

template <typename F>
double resolved_integral(const F& f, double lo, double hi) {
    long double p8, p16, q8, q16;
    composite(f, lo, hi, 1, p8, p16);
    for (std::size_t cells = 2; cells < (1u << 24); cells *= 2) {
        composite(f, lo, hi, cells, q8, q16);
        const double v = static_cast<double>(q16);
        const long double sp = spacing(v);
        if (std::fabs(q16 - q8) <= sp && std::fabs(q16 - p16) <= sp) return v;
        p16 = q16;
    }
    throw std::overflow_error("quadrature did not resolve");
}

double log_ratio(double upper, double lower) {
    const double rel = (upper - lower) / lower;
    return std::isfinite(rel) ? std::log1p(rel) : std::log(upper) - std::log(lower);
}

// Integral over u = ln(a/base) of g(a) for a1 -> a2 (signed).
template <typename G>
double log_integral(double a1, double a2, const G& g) {
    const bool forward = a2 > a1;
    const double base = forward ? a1 : a2;
    const double upper = forward ? a2 : a1;
    const double width = log_ratio(upper, base);
    if (!(width > 0.0)) throw std::underflow_error("empty interval");
    const double v = resolved_integral(
        [&](double u) {
            const double r = std::exp(u);
            double a = base * r;
            if (!std::isfinite(a) || a <= 0.0) a = std::exp(std::log(base) + u);
            return g(a);
        },
        0.0, width);
    return forward ? v : -v;
}

// Correctly rounded sqrt(a*b) by exact integer arithmetic on the significands.
double geometric_mean_exact(double a, double b) {
    int ea, eb;
    const double fa = std::frexp(a, &ea);  // a = fa 2^ea, fa in [0.5,1)
    const double fb = std::frexp(b, &eb);
    const uint64_t ma = static_cast<uint64_t>(std::ldexp(fa, 53));  // exact, 53 bits
    const uint64_t mb = static_cast<uint64_t>(std::ldexp(fb, 53));
    // a*b = ma*mb * 2^(ea+eb-106)
    unsigned __int128 P = static_cast<unsigned __int128>(ma) * mb;  // < 2^106
    int e = ea + eb - 106;
    if (e & 1) {
        P <<= 1;
        e -= 1;
    }
    // Scale P by 4^k so that floor(sqrt(P')) has exactly 54 bits (53 + guard).
    int k = 0;
    auto bits = [](unsigned __int128 v) {
        int n = 0;
        while (v) {
            v >>= 1;
            ++n;
        }
        return n;
    };
    while (bits(P) < 107) {
        P <<= 2;
        ++k;
    }
    while (bits(P) > 108) {
        P >>= 2;  // never taken for products of 53-bit significands
        --k;
    }
    // s = floor(sqrt(P)): start from a long-double estimate and correct.
    uint64_t s = static_cast<uint64_t>(std::sqrt(static_cast<long double>(P)));
    while (static_cast<unsigned __int128>(s) * s > P) --s;
    while (static_cast<unsigned __int128>(s + 1) * (s + 1) <= P) ++s;
    const bool sticky = static_cast<unsigned __int128>(s) * s != P;
    int sb = 0;
    for (uint64_t t = s; t; t >>= 1) ++sb;
    // Reduce s to 54 bits (53 + guard), folding dropped bits into sticky.
    int drop = sb - 54;
    bool st = sticky;
    uint64_t g = s;
    if (drop > 0) {
        st = st || (g & ((1ull << drop) - 1)) != 0;
        g >>= drop;
    }
    uint64_t m = g >> 1;
    const bool guard = g & 1;
    if (guard && (st || (m & 1))) ++m;
    // value = m * 2^(drop+1) * 2^(e/2 - k)
    return std::ldexp(static_cast<double>(m), (drop > 0 ? drop : 0) + 1 + e / 2 - k);
}

}  // namespace

extern "C" {

int hyowon_hubble(double om, double ol, uint64_t n, const double* a, double* H) {
    if (!valid_cosmology(om, ol) || (n && (!a || !H))) return kInvalid;
    const Cosmo c(om, ol);
    for (uint64_t i = 0; i < n; ++i) {
        if (!std::isfinite(a[i]) || a[i] <= 0.0) return kInvalid;
        H[i] = c.H(a[i]);
        if (!std::isfinite(H[i])) return kOverflow;
    }
    return kOk;
}

int hyowon_drift_factor(double om, double ol, double a1, double a2, double* D) {
    if (!valid_cosmology(om, ol) || !D || !std::isfinite(a1) || !std::isfinite(a2) || a1 <= 0.0
        || a2 <= 0.0)
        return kInvalid;
    if (a1 == a2) {
        *D = 0.0;
        return kOk;
    }
    const Cosmo c(om, ol);
    try {
        *D = log_integral(a1, a2, [&](double a) { return 1.0 / (a * (a * c.H(a))); });
    } catch (...) {
        return kOverflow;
    }
    return std::isfinite(*D) ? kOk : kOverflow;
}

int hyowon_kick_factor(double om, double ol, double a1, double a2, double* K) {
    if (!valid_cosmology(om, ol) || !K || !std::isfinite(a1) || !std::isfinite(a2) || a1 <= 0.0
        || a2 <= 0.0)
        return kInvalid;
    if (a1 == a2) {
        *K = 0.0;
        return kOk;
    }
    const Cosmo c(om, ol);
    try {
        *K = log_integral(a1, a2, [&](double a) { return 1.0 / (a * c.H(a)); });
    } catch (...) {
        return kOverflow;
    }
    return std::isfinite(*K) ? kOk : kOverflow;
}

int hyowon_geometric_mean(double a, double b, double* out) {
    if (!out || !std::isfinite(a) || !std::isfinite(b) || a <= 0.0 || b <= 0.0) return kInvalid;
    *out = geometric_mean_exact(a, b);
    return kOk;
}

int hyowon_schedule(double om, double ol, double a_start, double a_final, double dlna,
                    uint64_t max_steps, double* out6, uint64_t* n_steps) {
    if (!valid_cosmology(om, ol) || !n_steps || !std::isfinite(a_start) || !std::isfinite(a_final)
        || !std::isfinite(dlna) || a_start <= 0.0 || a_final <= 0.0 || dlna <= 0.0
        || a_start > a_final)
        return kInvalid;
    *n_steps = 0;
    if (a_start == a_final) return kOk;
    const double span = log_ratio(a_final, a_start);
    const double ratio = span / dlna;
    const double count_real =
        std::fmax(1.0, std::ceil(std::nextafter(ratio, std::numeric_limits<double>::infinity())));
    const uint64_t count = static_cast<uint64_t>(count_real);
    // Boundaries a_k = fma(a0, expm1(k dlna), a0) below the stop, then the stop.
    double prev = a_start;
    uint64_t k_out = 0;
    auto emit = [&](double next) -> int {
        if (!(next > prev)) return kOverflow;
        if (k_out >= max_steps) return kInvalid;
        double half;
        hyowon_geometric_mean(prev, next, &half);
        if (!(half > prev && half < next)) return kOverflow;
        if (out6) {
            double* r = out6 + 6 * k_out;
            r[0] = prev;
            r[1] = half;
            r[2] = next;
            int rc = hyowon_drift_factor(om, ol, prev, next, &r[3]);
            rc |= hyowon_kick_factor(om, ol, prev, half, &r[4]);
            rc |= hyowon_kick_factor(om, ol, half, next, &r[5]);
            if (rc) return kOverflow;
        }
        ++k_out;
        prev = next;
        return kOk;
    };
    for (uint64_t k = 1; k < count; ++k) {
        const double offset = dlna * static_cast<double>(k);
        const double rel = std::expm1(offset);
        const double next = std::isfinite(rel) ? std::fma(a_start, rel, a_start)
                                               : std::exp(std::log(a_start) + offset);
        if (next >= a_final) break;
        double tail_half;
        hyowon_geometric_mean(next, a_final, &tail_half);
        if (!(tail_half > next && tail_half < a_final)) break;
        const int rc = emit(next);
        if (rc) return rc;
    }
    const int rc = emit(a_final);
    if (rc) return rc;
    *n_steps = k_out;
    return kOk;
}

int hyowon_growth(double om, double ol, uint64_t n, const double* a, double* D1, double* f1) {
    if (!valid_cosmology(om, ol) || (n && (!a || !D1 || !f1))) return kInvalid;
    const Cosmo c(om, ol);
    // I(a) = int_0^a da'/(a'E)^3 with a' = s^(2/5): smooth integrand in s.
    auto I = [&](double a_end) {
        const double s_end = std::pow(a_end, 2.5);
        return resolved_integral(
            [&](double s) {
                const double ap = std::pow(s, 0.4);
                const double aE = ap * c.E(ap);
                return 0.4 * std::pow(s, -0.6) / (aE * aE * aE);
            },
            0.0, s_end);
    };
    try {
        const double I1 = I(1.0);
        const double Dnorm = c.E(1.0) * I1;
        for (uint64_t i = 0; i < n; ++i) {
            if (!std::isfinite(a[i]) || a[i] <= 0.0) return kInvalid;
            const double ai = a[i];
            const double Ii = I(ai);
            const double Ei = c.E(ai);
            D1[i] = Ei * Ii / Dnorm;
            const double dlnE = -1.5 * om / (ai * ai * ai * Ei * Ei);
            f1[i] = dlnE + 1.0 / (Ii * ai * ai * Ei * Ei * Ei);
        }
    } catch (...) {
        return kOverflow;
    }
    return kOk;
}

// Second-order growth (include/cosmo_nbody/cosmology/cosmology_model.hpp:50-53,
// src/cosmology/cosmology_model.cpp:194-320): y = [D1, dD1/dx, D2, dD2/dx] in
// x = ln a obeys y0' = y1, y1' = -(2 - 3/2 Om(a)) y1 + 3/2 Om(a) y0,
// y2' = y3, y3' = -(2 - 3/2 Om(a)) y3 + 3/2 Om(a) (y2 - y0^2), started in the
// matter era at a_s = (eps Om / OL)^(1/3) from the EdS growing modes
// (a, a, -3/7 a^2, -6/7 a^2) and integrated by classical RK4 with steps
// <= eps^(1/5) / 2 in ln a (the reference's balanced step, refined once).
// Normalised by D1(1) and D1(1)^2; f2 = y3 / y2. D1 and f1 come from
// hyowon_growth's integral solution.
int hyowon_growth2(double om, double ol, uint64_t n, const double* a, double* D1, double* f1,
                   double* D2, double* f2) {
    if (!valid_cosmology(om, ol) || (n && (!a || !D1 || !f1 || !D2 || !f2))) return kInvalid;
    for (uint64_t i = 0; i < n; ++i)
        if (!std::isfinite(a[i]) || a[i] <= 0.0 || a[i] > 1.0) return kInvalid;
    if (int rc = hyowon_growth(om, ol, n, a, D1, f1)) return rc;
    if (ol == 0.0) {
        for (uint64_t i = 0; i < n; ++i) {
            D2[i] = -3.0 / 7.0 * a[i] * a[i];
            f2[i] = 2.0;
        }
        return kOk;
    }
    const double eps = std::numeric_limits<double>::epsilon();
    const double a_s = std::fmin(std::cbrt(eps * om / ol), 1.0);
    const double x0 = std::log(a_s);
    const double h_max = 0.5 * std::pow(eps, 0.2);
    auto om_a = [&](double x) {
        const double a3 = std::exp(3.0 * x);
        return om / (om + ol * a3);
    };
    auto rhs = [&](double x, const double* y, double* d) {
        const double m = om_a(x);
        const double drag = 2.0 - 1.5 * m;
        d[0] = y[1];
        d[1] = -drag * y[1] + 1.5 * m * y[0];
        d[2] = y[3];
        d[3] = -drag * y[3] + 1.5 * m * y[2] - 1.5 * m * y[0] * y[0];
    };
    // state at ln a = x1
    auto integrate = [&](double x1, double* y) {
        y[0] = a_s;
        y[1] = a_s;
        y[2] = -(3.0 / 7.0) * a_s * a_s;
        y[3] = -(6.0 / 7.0) * a_s * a_s;
        if (!(x1 > x0)) return;
        const uint64_t steps = static_cast<uint64_t>(std::ceil((x1 - x0) / h_max));
        const double h = (x1 - x0) / static_cast<double>(steps);
        double k1[4], k2[4], k3[4], k4[4], t[4];
        for (uint64_t s = 0; s < steps; ++s) {
            const double x = x0 + static_cast<double>(s) * h;
            rhs(x, y, k1);
            for (int j = 0; j < 4; ++j) t[j] = y[j] + 0.5 * h * k1[j];
            rhs(x + 0.5 * h, t, k2);
            for (int j = 0; j < 4; ++j) t[j] = y[j] + 0.5 * h * k2[j];
            rhs(x + 0.5 * h, t, k3);
            for (int j = 0; j < 4; ++j) t[j] = y[j] + h * k3[j];
            rhs(x + h, t, k4);
            for (int j = 0; j < 4; ++j) y[j] += (h / 6.0) * (k1[j] + 2.0 * k2[j] + 2.0 * k3[j] + k4[j]);
        }
    };
    double y1[4];
    integrate(0.0, y1);
    const double d1_today = y1[0];
    if (!std::isfinite(d1_today) || d1_today <= 0.0) return kOverflow;
    for (uint64_t i = 0; i < n; ++i) {
        double y[4];
        const double x = std::log(a[i]);
        if (x <= x0) {
            const double r = a[i] / a_s;
            D2[i] = -(3.0 / 7.0) * a_s * a_s * r * r / (d1_today * d1_today);
            f2[i] = 2.0;
            continue;
        }
        integrate(x, y);
        D2[i] = y[2] / (d1_today * d1_today);
        f2[i] = y[3] / y[2];
        if (!std::isfinite(D2[i]) || !std::isfinite(f2[i]) || D2[i] >= 0.0) return kOverflow;
    }
    return kOk;
}

}  // extern "C"
