// Oracle: a CPU restatement of gw_fopt's generalized bulk-flow spectrum.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product links, imports or calls
// this file: it is the checker used by tests/, by __graft_entry__.smoke() and
// by the CPU-baseline leg of bench.py.  It restates, in plain f64 C++, the
// reference crate `bubble-gw` (Rust):
//
//   rust/bubble-gw/src/many_bubbles/generalized_bulk_flow.rs   (GBF)
//   rust/bubble-gw/src/many_bubbles/lattice_bubbles.rs         (LB)
//   rust/bubble-gw/src/many_bubbles/spacetime.rs               (Minkowski scalar)
//   rust/bubble-gw/src/time_cutoff.rs
//
// Parity status: UNPINNED against reference-produced numbers.  The reference
// crate cannot be built here (no Rust toolchain, its 183 crates are not
// vendored) and the only golden file its tests read
// (rust/bubble-gw/tests/envelope_2bubbles_scan=n_phix.csv) is absent from the
// snapshot.  The restatement is pinned instead by known-answer tests derived
// from the discretised mathematics (tests/test_oracle_kat.py) and by following
// the reference's arithmetic operation by operation:
//   * compiled with -ffp-contract=off (Rust never contracts a*b+c);
//   * glibc sin/cos/pow/exp/sqrt (Rust's f64 methods call the platform libm);
//   * nalgebra's 4-vector dot summed left to right ((p0+p1)+p2)+p3;
//   * ndarray's linspace a + step*i and its eight-way unrolled `sum`.
// The one deliberate difference: the reference reduces over t with a rayon
// fold whose order is not deterministic (GBF:811-866); this file sums t in
// index order so that it is reproducible for any thread count.

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include <algorithm>
#include <atomic>
#include <thread>

namespace {

// Dynamic parallel-for over [0, n) with `threads` workers; each worker owns
// one scratch object.  Work items are independent, so results do not depend
// on the thread count.
template <class Scratch, class F>
void parallel_for(size_t n, int threads, F&& f) {
    int nt = threads > 0 ? threads : 1;
    if ((size_t)nt > n) nt = (int)std::max<size_t>(n, 1);
    std::atomic<size_t> next{0};
    auto worker = [&]() {
        Scratch sc{};
        for (;;) {
            size_t i = next.fetch_add(1);
            if (i >= n) break;
            f(i, sc);
        }
    };
    if (nt == 1) {
        worker();
        return;
    }
    std::vector<std::thread> pool;
    for (int k = 0; k < nt; ++k) pool.emplace_back(worker);
    for (auto& th : pool) th.join();
}

struct V4 {
    double t, x, y, z;
};

// spacetime.rs:593-600: scalar(a, b) = dual(a).dot(b), dual negates the time
// component; nalgebra's fixed-size U4 dot is a + b + c + d, left to right.
inline double mdot(const V4& a, const V4& b) {
    double p0 = (-a.t) * b.t;
    double p1 = a.x * b.x;
    double p2 = a.y * b.y;
    double p3 = a.z * b.z;
    return ((p0 + p1) + p2) + p3;
}

inline V4 sub(const V4& b, const V4& a) { return V4{b.t - a.t, b.x - a.x, b.y - a.y, b.z - a.z}; }

// ndarray Array1::linspace: step = (b - a) / (n - 1); x_i = a + step * i.
std::vector<double> linspace(double a, double b, size_t n) {
    std::vector<double> v(n);
    double step = n > 1 ? (b - a) / (double)(n - 1) : 0.0;
    for (size_t i = 0; i < n; ++i) v[i] = a + step * (double)i;
    return v;
}

// ndarray's ArrayBase::sum for contiguous data: numeric_util::unrolled_fold
// with eight partial accumulators (ndarray 0.17, src/numeric_util.rs).
double unrolled_sum(const double* xs, size_t n) {
    double acc = 0.0;
    double p0 = 0, p1 = 0, p2 = 0, p3 = 0, p4 = 0, p5 = 0, p6 = 0, p7 = 0;
    while (n >= 8) {
        p0 = p0 + xs[0]; p1 = p1 + xs[1]; p2 = p2 + xs[2]; p3 = p3 + xs[3];
        p4 = p4 + xs[4]; p5 = p5 + xs[5]; p6 = p6 + xs[6]; p7 = p7 + xs[7];
        xs += 8; n -= 8;
    }
    acc = acc + (p0 + p4);
    acc = acc + (p1 + p5);
    acc = acc + (p2 + p6);
    acc = acc + (p3 + p7);
    for (size_t i = 0; i < n && i < 7; ++i) acc = acc + xs[i];
    return acc;
}

struct Cplx {
    double re, im;
};
// num-complex 0.4.6 Mul: (a.re*b.re - a.im*b.im, a.re*b.im + a.im*b.re)
inline Cplx cmul(Cplx a, Cplx b) { return Cplx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline Cplx cadd(Cplx a, Cplx b) { return Cplx{a.re + b.re, a.im + b.im}; }
// Complex * f64 scalar: each component times the scalar.
inline Cplx cscale(Cplx a, double s) { return Cplx{a.re * s, a.im * s}; }
// num-complex exp of (re, im) with re == +0: from_polar(exp(0), im) = (cos im, sin im).
inline Cplx cexp_i(double im) { return Cplx{1.0 * std::cos(im), 1.0 * std::sin(im)}; }

const int32_t kNone = -1;  // BubbleIndex::None; interior i >= 0; exterior e -> -(e+2)

struct Problem {
    std::vector<V4> interior, exterior;
    size_t n_int = 0, n_tot = 0;
    size_t n_cos = 0, n_phi = 0;
    std::vector<double> cos_thetax, phix;
    std::vector<V4> dirs;  // (n_cos, n_phi), row-major
    size_t n_sets = 1, n_terms = 1;
    std::vector<double> coeffs{1.0}, powers{3.0};
    bool has_damping = false;
    double damping = 0.0;

    const V4& bubble(size_t b) const { return b < n_int ? interior[b] : exterior[b - n_int]; }
    // LB:273-297: delta[(a, b)] = x_b - x_a (the lower triangle stores the
    // negated upper one, which is bitwise the same value).
    V4 delta(size_t a, size_t b) const { return sub(bubble(b), interior[a]); }
};

// GBF:208-238 (set_resolution).
void set_resolution(Problem& P, size_t n_cos, size_t n_phi) {
    P.n_cos = n_cos;
    P.n_phi = n_phi;
    P.cos_thetax = linspace(-1.0, 1.0, n_cos);
    P.phix = linspace(0.0, 2.0 * M_PI, n_phi);
    P.dirs.resize(n_cos * n_phi);
    for (size_t i = 0; i < n_cos; ++i) {
        double c = P.cos_thetax[i];
        double s = std::fabs(std::sqrt(1.0 - c * c));
        for (size_t j = 0; j < n_phi; ++j) {
            double phi = P.phix[j];
            double sp = std::sin(phi), cp = std::cos(phi);
            P.dirs[i * n_phi + j] = V4{1.0, s * cp, s * sp, c};
        }
    }
}

// GBF:1003-1018.
inline bool check_collision_point(const V4& dba, const V4& dca, const V4& x) {
    double dbx = mdot(dba, x);
    if (dbx <= 0.0) return false;
    double nb = mdot(dba, dba);
    double nc = mdot(dca, dca);
    V4 cv{dba.t * nc - dca.t * nb, dba.x * nc - dca.x * nb, dba.y * nc - dca.y * nb, dba.z * nc - dca.z * nb};
    return mdot(cv, x) > 0.0;
}

// GBF:127-206 for one direction.
int32_t first_colliding_one(const Problem& P, size_t a, const V4& x) {
    const double tol = 1e-10;
    int32_t best = kNone;
    double best_tau = std::numeric_limits<double>::infinity();
    for (size_t b = 0; b < P.n_tot; ++b) {
        if (b < P.n_int && b == a) continue;
        V4 dba = P.delta(a, b);
        double dsq = mdot(dba, dba);
        double dot = mdot(dba, x);
        if (dot <= tol) continue;
        double tau = dsq / (2.0 * dot);
        if (tau <= 0.0 || tau >= best_tau) continue;
        bool first = true;
        for (size_t c = 0; c < P.n_tot; ++c) {
            if ((c < P.n_int && c == a) || c == b) continue;
            V4 dca = P.delta(a, c);
            if (!check_collision_point(dba, dca, x)) {
                first = false;
                break;
            }
        }
        if (first) {
            best = b < P.n_int ? (int32_t)b : -((int32_t)(b - P.n_int) + 2);
            best_tau = tau;
        }
    }
    return best;
}

size_t decode_total(const Problem& P, int32_t code) {
    return code >= 0 ? (size_t)code : P.n_int + (size_t)(-code - 2);
}

// GBF:421-471.
void delta_tab(const Problem& P, size_t a, const int32_t* first, double* out) {
    for (size_t i = 0; i < P.n_cos; ++i)
        for (size_t j = 0; j < P.n_phi; ++j) {
            size_t k = i * P.n_phi + j;
            out[k] = 0.0;
            if (first[k] == kNone) continue;
            size_t b = decode_total(P, first[k]);
            V4 dba = P.delta(a, b);
            double dsq = mdot(dba, dba);
            double dot = mdot(dba, P.dirs[k]);
            if (std::fabs(dot) < 1e-10) {
                out[k] = 0.0;
                continue;
            }
            out[k] = dsq / (2.0 * dot);
        }
}

// time_cutoff.rs:15-43.
struct Cutoff {
    bool exponential = false;
    double t_cut = 0, t_0 = 0, inv_t_0_sq = 0;
    double eval(double t) const {
        if (!exponential) return 1.0;
        if (t < t_cut) return 1.0;
        double d = t - t_cut;
        double e = -(d * d) * inv_t_0_sq;
        return std::exp(e);
    }
};

Cutoff make_cutoff(int kind, double smax, double r_cut, double r_0) {
    Cutoff c;
    if (kind == 1) {
        c.exponential = true;
        double rc = std::isnan(r_cut) ? 0.999999999 : r_cut;
        double r0 = std::isnan(r_0) ? 0.25 : r_0;
        c.t_cut = rc * smax;
        c.t_0 = r0 * (smax - c.t_cut);
        c.inv_t_0_sq = 1.0 / (c.t_0 * c.t_0);
    }
    return c;
}

// GBF:369-414 (status), GBF:481-586 (B integral) for one cos(theta) row.
// status: 0 never, 1 already, 2 not yet.
void b_integral(const Problem& P, size_t i, const int32_t* first, const double* dtab, double delta_ta,
                double* b_plus, double* b_minus, std::vector<double>& scratch) {
    size_t nf = P.n_phi, S = P.n_sets, M = P.n_terms;
    for (size_t s = 0; s < S; ++s) b_plus[s] = b_minus[s] = 0.0;
    double c = P.cos_thetax[i];
    double sin_sq = 1.0 - c * c;
    double dphi = 2.0 * M_PI / (double)nf;
    if (delta_ta <= 0.0) return;
    double cubed = delta_ta * (delta_ta * delta_ta);
    scratch.resize(3 * nf);
    double* factors = scratch.data();
    double* cs = factors + nf;
    double* cc = cs + nf;
    for (size_t s = 0; s < S; ++s) {
        for (size_t j = 0; j < nf; ++j) {
            size_t k = i * nf + j;
            bool collided = false;
            if (first[k] != kNone) {
                double dt = dtab[k];
                collided = dt > 0.0 && delta_ta >= dt;
            }
            if (!collided) {
                factors[j] = 1.0;
            } else {
                double ratio = dtab[k] / delta_ta;
                double f = 0.0;
                for (size_t m = 0; m < M; ++m) f += P.coeffs[s * M + m] * std::pow(ratio, P.powers[s * M + m]);
                if (P.has_damping) {
                    double damp = std::exp(-delta_ta * (1.0 - ratio) / P.damping);
                    f *= damp;
                }
                factors[j] = f;
            }
        }
        for (size_t j = 0; j < nf; ++j) {
            double p = P.phix[j];
            double w = (j == 0 || j == nf - 1) ? 0.5 : 1.0;
            cs[j] = std::sin(2.0 * p) * factors[j] * w;
            cc[j] = std::cos(2.0 * p) * factors[j] * w;
        }
        double integral_minus = unrolled_sum(cs, nf) * dphi * cubed;
        double integral_plus = unrolled_sum(cc, nf) * dphi * cubed;
        b_plus[s] += 0.5 * sin_sq * integral_plus;
        b_minus[s] += 0.5 * sin_sq * integral_minus;
    }
}

// GBF:588-664 (A integral) followed by the per-t C increment of GBF:821-851.
// `inc` receives (2, S, W) complex values already multiplied by dt.  With
// `integrand` the tail is that of compute_c_integrand_fixed_bubble
// (GBF:820-840): A e^{i w (t - z_a)} (dt weight), no time cutoff.
void c_increment(const Problem& P, size_t a, const int32_t* first, const double* dtab, const double* w,
                 size_t W, double t, size_t t_idx, size_t n_t, double dt, const Cutoff& cut, Cplx* inc,
                 std::vector<double>& scratch, bool integrand = false) {
    size_t S = P.n_sets, nc = P.n_cos;
    double ta = P.interior[a].t, za = P.interior[a].z;
    double delta_ta = t - ta;
    std::vector<Cplx> ap(S * W, Cplx{0, 0}), am(S * W, Cplx{0, 0});
    std::vector<double> bp(S), bm(S);
    std::vector<Cplx> pf(W);
    double dcos = 2.0 / (double)(nc - 1);
    for (size_t i = 0; i < nc; ++i) {
        b_integral(P, i, first, dtab, delta_ta, bp.data(), bm.data(), scratch);
        double cval = P.cos_thetax[i];
        double base_im = -delta_ta * cval;
        double wt = (i == 0 || i == nc - 1) ? 0.5 : 1.0;
        for (size_t k = 0; k < W; ++k) {
            Cplx ph = cexp_i(w[k] * base_im);
            pf[k] = cscale(cscale(ph, dcos), wt);
        }
        for (size_t s = 0; s < S; ++s) {
            Cplx bps{bp[s], 0.0}, bms{bm[s], 0.0};
            for (size_t k = 0; k < W; ++k) {
                ap[s * W + k] = cadd(ap[s * W + k], cmul(bps, pf[k]));
                am[s * W + k] = cadd(am[s * W + k], cmul(bms, pf[k]));
            }
        }
    }
    double uw = (t_idx == 0 || t_idx == n_t - 1) ? 0.5 : 1.0;
    if (integrand) {
        Cplx dtw{dt * uw, 0.0};
        for (size_t s = 0; s < S; ++s)
            for (size_t k = 0; k < W; ++k) {
                Cplx ph = cexp_i(w[k] * (t - za));
                inc[(0 * S + s) * W + k] = cmul(cmul(ap[s * W + k], ph), dtw);
                inc[(1 * S + s) * W + k] = cmul(cmul(am[s * W + k], ph), dtw);
            }
        return;
    }
    double cw = cut.eval(t);
    Cplx dtc{dt, 0.0};
    for (size_t s = 0; s < S; ++s)
        for (size_t k = 0; k < W; ++k) {
            Cplx ph = cexp_i(w[k] * (t - za));
            Cplx ip = cscale(cscale(cmul(ap[s * W + k], ph), uw), cw);
            Cplx im = cscale(cscale(cmul(am[s * W + k], ph), uw), cw);
            inc[(0 * S + s) * W + k] = cmul(ip, dtc);
            inc[(1 * S + s) * W + k] = cmul(im, dtc);
        }
}

// ---- tensor form: new_generalized_bulk_flow.rs (NGBF) ----
// NGBF:592-727 (compute_b_tensor) for one cos(theta) row: the six components
// xx, xy, xz, yy, yz, zz of the phi integral of x_i x_j (t - t_n)^3 f.
void b_tensor(const Problem& P, size_t i, const int32_t* first, const double* dtab, double delta_ta, double* b6,
              std::vector<double>& scratch) {
    size_t nf = P.n_phi, S = P.n_sets, M = P.n_terms;
    double c = P.cos_thetax[i];
    double st = std::sqrt(std::max(1.0 - c * c, 0.0));
    double s2 = st * st, c2 = c * c, sc = st * c;
    double dphi = 2.0 * M_PI / (double)nf;
    double cubed = delta_ta > 0.0 ? (delta_ta * delta_ta) * delta_ta : 0.0;
    scratch.resize(7 * nf);
    double* factors = scratch.data();
    double* wk = factors + nf;  // 6 weighted rows
    for (size_t s = 0; s < S; ++s) {
        for (size_t j = 0; j < nf; ++j) {
            size_t k = i * nf + j;
            bool collided = false;  // NGBF:480-530: AlreadyCollided iff tau > 0 and delta_ta >= tau
            if (first[k] != kNone) {
                double dt = dtab[k];
                collided = dt > 0.0 && delta_ta >= dt;
            }
            if (!collided) {
                factors[j] = 1.0;
            } else {
                double ratio = dtab[k] / delta_ta;
                double f = 0.0;
                for (size_t m = 0; m < M; ++m) f += P.coeffs[s * M + m] * std::pow(ratio, P.powers[s * M + m]);
                if (P.has_damping) f *= std::exp(-delta_ta * (1.0 - ratio) / P.damping);
                factors[j] = f;
            }
        }
        for (size_t j = 0; j < nf; ++j) {
            double cp = std::cos(P.phix[j]), sp = std::sin(P.phix[j]);
            double w = (nf > 1 && (j == 0 || j == nf - 1)) ? 0.5 : 1.0;
            double basis[6] = {(cp * cp) * s2, (cp * sp) * s2, cp * sc, (sp * sp) * s2, sp * sc, c2};
            for (int q = 0; q < 6; ++q) wk[q * nf + j] = (basis[q] * factors[j]) * w;
        }
        for (int q = 0; q < 6; ++q) b6[q * S + s] = (unrolled_sum(wk + q * nf, nf) * dphi) * cubed;
    }
}

// NGBF:729-830 (compute_a_tensor) and the per-t increment of NGBF:1130-1168:
// inc (6, S, W) = A(t) e^{i w (t - z_a)} (dt weight).
void c_tensor_increment(const Problem& P, size_t a, const int32_t* first, const double* dtab, const double* w,
                        size_t W, double t, size_t t_idx, size_t n_t, double dt, Cplx* inc,
                        std::vector<double>& scratch) {
    size_t S = P.n_sets, nc = P.n_cos;
    double ta = P.interior[a].t, za = P.interior[a].z;
    double delta_ta = t - ta;
    std::vector<Cplx> acc(6 * S * W, Cplx{0, 0});
    std::vector<double> b6(6 * S);
    std::vector<Cplx> ph(W);
    double dcos = nc > 1 ? 2.0 / (double)(nc - 1) : 1.0;
    for (size_t i = 0; i < nc; ++i) {
        b_tensor(P, i, first, dtab, delta_ta, b6.data(), scratch);
        double base_im = -delta_ta * P.cos_thetax[i];
        double wt = nc == 1 ? 1.0 : ((i == 0 || i == nc - 1) ? 0.5 : 1.0);
        double pfs = dcos * wt;
        for (size_t k = 0; k < W; ++k) ph[k] = cscale(cexp_i(w[k] * base_im), pfs);
        for (int q = 0; q < 6; ++q)
            for (size_t s = 0; s < S; ++s) {
                Cplx bv{b6[q * S + s], 0.0};
                for (size_t k = 0; k < W; ++k)
                    acc[(q * S + s) * W + k] = cadd(acc[(q * S + s) * W + k], cmul(bv, ph[k]));
            }
    }
    double uw = (t_idx == 0 || t_idx == n_t - 1) ? 0.5 : 1.0;
    Cplx dtc{dt * uw, 0.0};
    for (size_t k = 0; k < W; ++k) {
        Cplx factor = cmul(cexp_i(w[k] * (t - za)), dtc);
        for (size_t q = 0; q < 6 * S; ++q) inc[q * W + k] = cmul(acc[q * W + k], factor);
    }
}

// NGBF:1067-1203 (compute_c_tensor_fixed_bubble), t reduced in index order; adds into acc (6, S, W).
void c_tensor_fixed_bubble(const Problem& P, size_t a, const int32_t* first, const double* w, size_t W,
                           double t_begin, double t_end, size_t n_t, Cplx* acc, int threads) {
    size_t S = P.n_sets;
    std::vector<double> dtab(P.n_cos * P.n_phi);
    delta_tab(P, a, first, dtab.data());
    std::vector<double> t_arr = linspace(t_begin, t_end, n_t);
    double dt = n_t > 1 ? t_arr[1] - t_arr[0] : 0.0;
    size_t per = 6 * S * W;
    std::vector<Cplx> incs(n_t * per, Cplx{0, 0});
    std::vector<char> active(n_t, 0);
    double tn = P.interior[a].t;
    parallel_for<std::vector<double>>(n_t, threads, [&](size_t ti, std::vector<double>& scratch) {
        double t = t_arr[ti];
        if (t > tn) {  // NGBF:1130: t <= t_nucleation contributes nothing
            active[ti] = 1;
            c_tensor_increment(P, a, first, dtab.data(), w, W, t, ti, n_t, dt, &incs[ti * per], scratch);
        }
    });
    std::vector<Cplx> c(per, Cplx{0, 0});
    for (size_t ti = 0; ti < n_t; ++ti)
        if (active[ti])
            for (size_t q = 0; q < per; ++q) c[q] = cadd(c[q], incs[ti * per + q]);
    Cplx f{1.0 / (6.0 * M_PI), 0.0};
    for (size_t q = 0; q < per; ++q) acc[q] = cadd(acc[q], cmul(c[q], f));
}

thread_local std::string g_err;

int fail(const std::string& m) {
    g_err = m;
    return 1;
}

void load(Problem& P, const double* interior, size_t n_int, const double* exterior, size_t n_ext) {
    P.interior.resize(n_int);
    P.exterior.resize(n_ext);
    for (size_t i = 0; i < n_int; ++i)
        P.interior[i] = V4{interior[4 * i], interior[4 * i + 1], interior[4 * i + 2], interior[4 * i + 3]};
    for (size_t i = 0; i < n_ext; ++i)
        P.exterior[i] = V4{exterior[4 * i], exterior[4 * i + 1], exterior[4 * i + 2], exterior[4 * i + 3]};
    P.n_int = n_int;
    P.n_tot = n_int + n_ext;
}

void set_params(Problem& P, const double* coeffs, const double* powers, size_t S, size_t M, double damping) {
    P.n_sets = S;
    P.n_terms = M;
    P.coeffs.assign(coeffs, coeffs + S * M);
    P.powers.assign(powers, powers + S * M);
    P.has_damping = !std::isnan(damping);
    P.damping = damping;
}

void masks_for(const Problem& P, size_t a, int32_t* out, int threads) {
    size_t nd = P.n_cos * P.n_phi;
    parallel_for<int>(nd, threads, [&](size_t k, int&) { out[k] = first_colliding_one(P, a, P.dirs[k]); });
}

// GBF:775-873 for one bubble, t reduced in index order; adds into `acc`.
void c_fixed_bubble(const Problem& P, size_t a, const int32_t* first, const double* w, size_t W, double t_begin,
                    double t_end, size_t n_t, const Cutoff& cut, Cplx* acc, double* abs_acc, int threads) {
    size_t S = P.n_sets;
    std::vector<double> dtab(P.n_cos * P.n_phi);
    delta_tab(P, a, first, dtab.data());
    std::vector<double> t_arr = linspace(t_begin, t_end, n_t);
    double dt = n_t > 1 ? t_arr[1] - t_arr[0] : 0.0;
    size_t per = 2 * S * W;
    std::vector<Cplx> incs(n_t * per, Cplx{0, 0});
    std::vector<char> active(n_t, 0);
    double tn = P.interior[a].t;
    parallel_for<std::vector<double>>(n_t, threads, [&](size_t ti, std::vector<double>& scratch) {
        double t = t_arr[ti];
        if (tn <= t) {
            active[ti] = 1;
            c_increment(P, a, first, dtab.data(), w, W, t, ti, n_t, dt, cut, &incs[ti * per], scratch);
        }
    });
    // Per-bubble fold in t order, then the 1/(6 pi) factor (GBF:867-869),
    // then accumulation into the total (GBF:971-981).
    std::vector<Cplx> c(per, Cplx{0, 0});
    for (size_t ti = 0; ti < n_t; ++ti) {
        if (!active[ti]) continue;
        for (size_t q = 0; q < per; ++q) {
            c[q] = cadd(c[q], incs[ti * per + q]);
            if (abs_acc) abs_acc[q] += std::hypot(incs[ti * per + q].re, incs[ti * per + q].im);
        }
    }
    Cplx f{1.0 / (6.0 * M_PI), 0.0};
    for (size_t q = 0; q < per; ++q) acc[q] = cadd(acc[q], cmul(c[q], f));
}

}  // namespace

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

// LB:71-119 and LB:273-297 for an EmptyLattice: causality of interior-interior
// and interior-exterior pairs.  Returns 0 when valid.
int orc_validate(const double* interior, size_t n_int, const double* exterior, size_t n_ext) {
    Problem P;
    load(P, interior, n_int, exterior, n_ext);
    for (size_t a = 0; a < n_int; ++a)
        for (size_t b = a + 1; b < n_int; ++b) {
            V4 d = P.delta(a, b);
            if (mdot(d, d) < 0.0)
                return fail("Bubble Interior(" + std::to_string(a) + ") is formed inside bubble Interior(" +
                            std::to_string(b) + ") at initial time (overlapping light cones)");
        }
    for (size_t a = 0; a < n_int; ++a)
        for (size_t e = 0; e < n_ext; ++e) {
            V4 d = P.delta(a, n_int + e);
            if (mdot(d, d) < 0.0)
                return fail("Bubble Interior(" + std::to_string(a) + ") is formed inside bubble Exterior(" +
                            std::to_string(e) + ") at initial time (overlapping light cones)");
        }
    return 0;
}

// GBF:208-270: the (n_cos, n_phi) direction table as (x, y, z) triples.
void orc_directions(size_t n_cos, size_t n_phi, double* out_xyz) {
    Problem P;
    set_resolution(P, n_cos, n_phi);
    for (size_t k = 0; k < n_cos * n_phi; ++k) {
        out_xyz[3 * k] = P.dirs[k].x;
        out_xyz[3 * k + 1] = P.dirs[k].y;
        out_xyz[3 * k + 2] = P.dirs[k].z;
    }
}

// GBF:127-206 for interior bubbles [a_begin, a_end): out is (a_end-a_begin, n_cos, n_phi)
// int32 with the PyO3 encoding -1 = None, i = Interior(i), -(i+2) = Exterior(i)
// (rust/py-bubble-gw/src/py_many_bubbles/py_generalized_bulk_flow.rs:241-245).
int orc_first_colliding(const double* interior, size_t n_int, const double* exterior, size_t n_ext, size_t n_cos,
                        size_t n_phi, size_t a_begin, size_t a_end, int32_t* out, double* out_delta_tab,
                        int threads) {
    if (n_cos < 2 || n_phi < 2) return fail("Invalid resolution: Angular resolutions must be greater than one");
    Problem P;
    load(P, interior, n_int, exterior, n_ext);
    set_resolution(P, n_cos, n_phi);
    size_t nd = n_cos * n_phi;
    for (size_t a = a_begin; a < a_end; ++a) {
        int32_t* o = out + (a - a_begin) * nd;
        masks_for(P, a, o, threads);
        if (out_delta_tab) delta_tab(P, a, o, out_delta_tab + (a - a_begin) * nd);
    }
    return 0;
}

// GBF:928-984 through the C ABI's argument conventions
// (rust/c-bubble-gw/src/lib.rs:496-574).  `selected` NULL = all interior
// bubbles.  out: (2, n_sets, n_w) complex128 as interleaved doubles.
// abs_out (optional): sum over (bubble, t) of |increment| per output entry,
// for the condition number kappa = abs_out / |out|.
int orc_compute_c_integral(const double* interior, size_t n_int, const double* exterior, size_t n_ext,
                           size_t n_cos, size_t n_phi, const double* coeffs, const double* powers, size_t n_sets,
                           size_t n_terms, double damping, const double* w, size_t n_w, int has_t_begin,
                           double t_begin, double t_end, size_t n_t, const size_t* selected, size_t n_sel,
                           int cutoff_kind, double smax, double ratio_t_cut, double ratio_t_0, double* out,
                           double* abs_out, int threads) {
    if (n_cos < 2 || n_phi < 2) return fail("Invalid resolution: Angular resolutions must be greater than one");
    Problem P;
    load(P, interior, n_int, exterior, n_ext);
    set_resolution(P, n_cos, n_phi);
    set_params(P, coeffs, powers, n_sets, n_terms, damping);
    size_t per = 2 * n_sets * n_w;
    std::vector<Cplx> acc(per, Cplx{0, 0});
    std::vector<double> absacc(per, 0.0);
    if (n_t < 2) return fail("Invalid resolution: n_t must be >= 2 for integration");
    std::vector<size_t> ids;
    if (selected) {
        for (size_t q = 0; q < n_sel; ++q) {
            if (selected[q] >= n_int)
                return fail("Index " + std::to_string(selected[q]) + " out of bounds for max " + std::to_string(n_int));
            ids.push_back(selected[q]);
        }
    } else {
        for (size_t a = 0; a < n_int; ++a) ids.push_back(a);
    }
    double tb = has_t_begin ? t_begin : 0.0;
    Cutoff cut = make_cutoff(cutoff_kind, smax, ratio_t_cut, ratio_t_0);
    std::vector<int32_t> first(n_cos * n_phi);
    for (size_t a : ids) {
        if (tb > t_end) return fail("Invalid time range");
        masks_for(P, a, first.data(), threads);
        c_fixed_bubble(P, a, first.data(), w, n_w, tb, t_end, n_t, cut, acc.data(), absacc.data(), threads);
    }
    for (size_t q = 0; q < per; ++q) {
        out[2 * q] = acc[q].re;
        out[2 * q + 1] = acc[q].im;
        if (abs_out) abs_out[q] = absacc[q] / (6.0 * M_PI);
    }
    return 0;
}

// compute_c_integrand (GBF:875-920) over compute_c_integrand_fixed_bubble
// (GBF:776-866): out (2, S, W, T) complex as interleaved doubles, the sum over
// the selected bubbles in selection order of each bubble's time-resolved
// integrand (already multiplied by the trapezoid dt weight and 1/(6 pi)).
int orc_compute_c_integrand(const double* interior, size_t n_int, const double* exterior, size_t n_ext,
                            size_t n_cos, size_t n_phi, const double* coeffs, const double* powers, size_t n_sets,
                            size_t n_terms, double damping, const double* w, size_t n_w, int has_t_begin,
                            double t_begin, double t_end, size_t n_t, const size_t* selected, size_t n_sel,
                            double* out, int threads) {
    if (n_cos < 2 || n_phi < 2) return fail("Invalid resolution: Angular resolutions must be greater than one");
    if (n_t < 2) return fail("Invalid resolution: n_t must be >= 2");
    Problem P;
    load(P, interior, n_int, exterior, n_ext);
    set_resolution(P, n_cos, n_phi);
    set_params(P, coeffs, powers, n_sets, n_terms, damping);
    const size_t S = n_sets, W = n_w, per = 2 * S * W;
    std::vector<Cplx> total(per * n_t, Cplx{0, 0});
    std::vector<size_t> ids;
    if (selected) {
        for (size_t q = 0; q < n_sel; ++q) {
            if (selected[q] >= n_int)
                return fail("Index " + std::to_string(selected[q]) + " out of bounds for max " + std::to_string(n_int));
            ids.push_back(selected[q]);
        }
    } else {
        for (size_t a = 0; a < n_int; ++a) ids.push_back(a);
    }
    double tb = has_t_begin ? t_begin : 0.0;
    Cutoff unit = make_cutoff(0, 0.0, NAN, NAN);
    std::vector<int32_t> first(n_cos * n_phi);
    std::vector<double> dtab(n_cos * n_phi);
    Cplx f{1.0 / (6.0 * M_PI), 0.0};
    for (size_t a : ids) {
        const double tn = P.interior[a].t;
        if (tn >= t_end) continue;  // GBF:786-789
        if (tb > t_end) return fail("Invalid time range");
        masks_for(P, a, first.data(), threads);
        delta_tab(P, a, first.data(), dtab.data());
        std::vector<double> t_arr = linspace(tb, t_end, n_t);
        const double dt = t_arr[1] - t_arr[0];
        std::vector<Cplx> incs(n_t * per, Cplx{0, 0});
        parallel_for<std::vector<double>>(n_t, threads, [&](size_t ti, std::vector<double>& scratch) {
            const double t = t_arr[ti];
            if (t <= tn) return;  // GBF:818-822
            c_increment(P, a, first.data(), dtab.data(), w, W, t, ti, n_t, dt, unit, &incs[ti * per], scratch,
                        true);
        });
        for (size_t ti = 0; ti < n_t; ++ti)
            for (size_t q = 0; q < per; ++q)
                total[q * n_t + ti] = cadd(total[q * n_t + ti], cmul(incs[ti * per + q], f));
    }
    for (size_t q = 0; q < per * n_t; ++q) {
        out[2 * q] = total[q].re;
        out[2 * q + 1] = total[q].im;
    }
    return 0;
}

// The k-hat convention shared by the oracle and the product: R maps k-hat to
// z-hat; it is the Rodrigues rotation about k x z (normalised) by
// acos(k . z); identity for k = +z, a pi rotation about x for k = -z.
// Entries are formed with this exact operation sequence (row-major R).
void orc_rotation_for_khat(double kx, double ky, double kz, double* R) {
    double ax = ky, ay = -kx;  // k x z = (ky, -kx, 0)
    double s2 = ax * ax + ay * ay;
    if (s2 < 1e-30) {
        double sgn = kz >= 0.0 ? 1.0 : -1.0;
        R[0] = 1.0; R[1] = 0.0; R[2] = 0.0;
        R[3] = 0.0; R[4] = sgn; R[5] = 0.0;
        R[6] = 0.0; R[7] = 0.0; R[8] = sgn;
        return;
    }
    double s = std::sqrt(s2);
    double ux = ax / s, uy = ay / s;
    double c = kz;
    double v = 1.0 - c;
    // R = c I + s [u]x + v u u^T with u = (ux, uy, 0)
    R[0] = c + v * (ux * ux);
    R[1] = v * (ux * uy);
    R[2] = s * uy;
    R[3] = v * (uy * ux);
    R[4] = c + v * (uy * uy);
    R[5] = -(s * ux);
    R[6] = -(s * uy);
    R[7] = s * ux;
    R[8] = c;
}

// Rotates (n, 4) [t, x, y, z] rows about the origin: x'_i = (R_i0 x + R_i1 y) + R_i2 z.
void orc_rotate(const double* R, const double* in, size_t n, double* out) {
    for (size_t q = 0; q < n; ++q) {
        double x = in[4 * q + 1], y = in[4 * q + 2], z = in[4 * q + 3];
        out[4 * q] = in[4 * q];
        out[4 * q + 1] = (R[0] * x + R[1] * y) + R[2] * z;
        out[4 * q + 2] = (R[3] * x + R[4] * y) + R[5] * z;
        out[4 * q + 3] = (R[6] * x + R[7] * y) + R[8] * z;
    }
}

// One spectrum per k-hat: the configuration (interior and exterior) is rotated
// with orc_rotation_for_khat and orc_compute_c_integral runs on the rotated
// arrays.  out: (K, 2, n_sets, n_w) complex128 interleaved.
int orc_compute_c_integral_khat(const double* interior, size_t n_int, const double* exterior, size_t n_ext,
                                const double* khat, size_t K, size_t n_cos, size_t n_phi, const double* coeffs,
                                const double* powers, size_t n_sets, size_t n_terms, double damping, const double* w,
                                size_t n_w, double t_begin, double t_end, size_t n_t, int cutoff_kind, double smax,
                                double ratio_t_cut, double ratio_t_0, double* out, int threads) {
    std::vector<double> ri(4 * n_int), re(4 * n_ext);
    double R[9];
    size_t per = 2 * n_sets * n_w;
    for (size_t k = 0; k < K; ++k) {
        orc_rotation_for_khat(khat[3 * k], khat[3 * k + 1], khat[3 * k + 2], R);
        orc_rotate(R, interior, n_int, ri.data());
        orc_rotate(R, exterior, n_ext, re.data());
        int rc = orc_compute_c_integral(ri.data(), n_int, re.data(), n_ext, n_cos, n_phi, coeffs, powers, n_sets,
                                        n_terms, damping, w, n_w, 1, t_begin, t_end, n_t, nullptr, 0, cutoff_kind,
                                        smax, ratio_t_cut, ratio_t_0, out + 2 * k * per, nullptr, threads);
        if (rc) return rc;
    }
    return 0;
}

// NGBF:1205-1275 (compute_c_tensor): out (6, S, W) complex as interleaved
// doubles, the sum over the selected bubbles (NULL = all) in selection order.
int orc_compute_c_tensor(const double* interior, size_t n_int, const double* exterior, size_t n_ext, size_t n_cos,
                         size_t n_phi, const double* coeffs, const double* powers, size_t n_sets, size_t n_terms,
                         double damping, const double* w, size_t n_w, int has_t_begin, double t_begin, double t_end,
                         size_t n_t, const size_t* selected, size_t n_sel, double* out, int threads) {
    if (n_cos < 2 || n_phi < 2) return fail("Invalid resolution: Angular resolutions must be greater than one");
    if (n_t < 2) return fail("Invalid resolution: n_t must be >= 2 for integration");
    Problem P;
    load(P, interior, n_int, exterior, n_ext);
    set_resolution(P, n_cos, n_phi);
    set_params(P, coeffs, powers, n_sets, n_terms, damping);
    size_t per = 6 * n_sets * n_w;
    std::vector<Cplx> acc(per, Cplx{0, 0});
    std::vector<size_t> ids;
    if (selected) {
        for (size_t q = 0; q < n_sel; ++q) {
            if (selected[q] >= n_int)
                return fail("Index " + std::to_string(selected[q]) + " out of bounds for max " + std::to_string(n_int));
            ids.push_back(selected[q]);
        }
    } else {
        for (size_t a = 0; a < n_int; ++a) ids.push_back(a);
    }
    double tb = has_t_begin ? t_begin : 0.0;
    if (tb > t_end) return fail("Invalid time range");
    std::vector<int32_t> first(n_cos * n_phi);
    for (size_t a : ids) {
        masks_for(P, a, first.data(), threads);
        c_tensor_fixed_bubble(P, a, first.data(), w, n_w, tb, t_end, n_t, acc.data(), threads);
    }
    for (size_t q = 0; q < per; ++q) {
        out[2 * q] = acc[q].re;
        out[2 * q + 1] = acc[q].im;
    }
    return 0;
}

// time_cutoff.rs:15-43 evaluated at n points.
void orc_time_cutoff(int kind, double smax, double r_cut, double r_0, const double* t, size_t n, double* out) {
    Cutoff c = make_cutoff(kind, smax, r_cut, r_0);
    for (size_t q = 0; q < n; ++q) out[q] = c.eval(t[q]);
}

int orc_max_threads(void) {
    unsigned n = std::thread::hardware_concurrency();
    return n ? (int)n : 1;
}

}  // extern "C"
