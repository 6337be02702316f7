// Host-side geometry: lattice containment, boundary images, causality
// validation, the angular/time grids and the k-hat rotation.
//
// Compiled with -ffp-contract=off: every expression below is evaluated in the
// operation order written, as the reference's Rust code is (Rust never fuses
// a*b+c), so that images and grids are bitwise those of the reference.

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "bgw_internal.h"

namespace bgw {

std::string rust_f64(double x) {
    if (std::isnan(x)) return "NaN";
    if (std::isinf(x)) return x > 0 ? "inf" : "-inf";
    if (x == 0.0) return std::signbit(x) ? "-0" : "0";
    // Shortest decimal mantissa that round-trips.
    char buf[64];
    int prec = 1;
    for (; prec <= 17; ++prec) {
        std::snprintf(buf, sizeof buf, "%.*e", prec - 1, x);
        if (std::strtod(buf, nullptr) == x) break;
    }
    // buf = [-]d.ddddde[+-]XX
    std::string s(buf);
    bool neg = s[0] == '-';
    if (neg) s = s.substr(1);
    size_t epos = s.find('e');
    int exp10 = std::atoi(s.c_str() + epos + 1);
    std::string digits;
    for (size_t q = 0; q < epos; ++q)
        if (s[q] != '.') digits += s[q];
    while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
    // value = 0.digits * 10^(exp10+1)
    int point = exp10 + 1;  // digits before the decimal point
    std::string out;
    if (point <= 0) {
        out = "0." + std::string((size_t)(-point), '0') + digits;
    } else if ((size_t)point >= digits.size()) {
        out = digits + std::string((size_t)point - digits.size(), '0');
    } else {
        out = digits.substr(0, (size_t)point) + "." + digits.substr((size_t)point);
    }
    return neg ? "-" + out : out;
}

// ndarray Array1::linspace (x_i = a + step*i, step = (b-a)/(n-1)).
std::vector<double> linspace(double a, double b, size_t n) {
    std::vector<double> v(n);
    double step = n > 1 ? (b - a) / (double)(n - 1) : 0.0;
    for (size_t i = 0; i < n; ++i) v[i] = a + step * (double)i;
    return v;
}

// R maps k-hat to z-hat: Rodrigues rotation about k x z (normalised) by
// acos(k.z); identity for +z, a pi rotation about x for -z.
void rotation_for_khat(double kx, double ky, double kz, double* R) {
    double ax = ky, ay = -kx;
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

namespace {

struct P3 {
    double x, y, z;
};
inline P3 sub3(P3 a, P3 b) { return P3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline double dot3(P3 a, P3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline P3 scale3(P3 a, double s) { return P3{a.x * s, a.y * s, a.z * s}; }
inline P3 neg3(P3 a) { return P3{-a.x, -a.y, -a.z}; }

// Inverse of the 3x3 matrix with columns e1, e2, e3 by cofactors; false when
// the determinant is zero (parallelepiped_lattice.rs:161-166).
bool inverse3(const double* e, double inv[3][3]) {
    // m[r][c] = e_c[r]
    double m[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) m[r][c] = e[3 * c + r];
    double c00 = m[1][1] * m[2][2] - m[2][1] * m[1][2];
    double c01 = m[1][0] * m[2][2] - m[2][0] * m[1][2];
    double c02 = m[1][0] * m[2][1] - m[2][0] * m[1][1];
    double det = m[0][0] * c00 - m[0][1] * c01 + m[0][2] * c02;
    if (det == 0.0) return false;
    inv[0][0] = c00 / det;
    inv[0][1] = -(m[0][1] * m[2][2] - m[2][1] * m[0][2]) / det;
    inv[0][2] = (m[0][1] * m[1][2] - m[1][1] * m[0][2]) / det;
    inv[1][0] = -c01 / det;
    inv[1][1] = (m[0][0] * m[2][2] - m[2][0] * m[0][2]) / det;
    inv[1][2] = -(m[0][0] * m[1][2] - m[1][0] * m[0][2]) / det;
    inv[2][0] = c02 / det;
    inv[2][1] = -(m[0][0] * m[2][1] - m[2][0] * m[0][1]) / det;
    inv[2][2] = (m[0][0] * m[1][1] - m[1][0] * m[0][1]) / det;
    return true;
}

inline double norm3(P3 a) { return std::sqrt(dot3(a, a)); }

}  // namespace

void lattice_contains(BgwxLatticeKind kind, const double* params, const double* pts, size_t n, uint8_t* out) {
    switch (kind) {
        case BGWX_LATTICE_PARALLELEPIPED:
        case BGWX_LATTICE_CARTESIAN: {
            double inv[3][3];
            if (!inverse3(params + 3, inv)) {
                for (size_t q = 0; q < n; ++q) out[q] = 0;
                return;
            }
            P3 o{params[0], params[1], params[2]};
            for (size_t q = 0; q < n; ++q) {
                P3 d = sub3(P3{pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]}, o);
                bool in = true;
                for (int r = 0; r < 3; ++r) {
                    double u = (inv[r][0] * d.x + inv[r][1] * d.y) + inv[r][2] * d.z;
                    in = in && u >= 0.0 && u <= 1.0;
                }
                out[q] = in ? 1 : 0;
            }
            return;
        }
        case BGWX_LATTICE_SPHERICAL: {
            P3 c{params[0], params[1], params[2]};
            double r2 = params[3] * params[3];
            for (size_t q = 0; q < n; ++q) {
                P3 d = sub3(P3{pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]}, c);
                out[q] = dot3(d, d) <= r2 ? 1 : 0;
            }
            return;
        }
        case BGWX_LATTICE_EMPTY:
        default:
            return;
    }
}

std::vector<double> lattice_exterior(BgwxLatticeKind kind, const double* params, BgwxBoundaryCondition bc,
                                     const double* interior, size_t n) {
    std::vector<double> out;
    if (bc == BGWX_BC_NONE || kind == BGWX_LATTICE_EMPTY) return out;
    auto push = [&](double t, P3 p) {
        out.push_back(t);
        out.push_back(p.x);
        out.push_back(p.y);
        out.push_back(p.z);
    };
    if (kind == BGWX_LATTICE_PARALLELEPIPED || kind == BGWX_LATTICE_CARTESIAN) {
        P3 o{params[0], params[1], params[2]};
        P3 e[3] = {{params[3], params[4], params[5]}, {params[6], params[7], params[8]}, {params[9], params[10], params[11]}};
        if (bc == BGWX_BC_PERIODIC) {
            // parallelepiped_lattice.rs:197-215: shifts +e1, -e1, +e2, -e2, +e3, -e3
            P3 shifts[6] = {e[0], neg3(e[0]), e[1], neg3(e[1]), e[2], neg3(e[2])};
            out.reserve(n * 24);
            for (size_t q = 0; q < n; ++q) {
                const double* ev = interior + 4 * q;
                for (auto& sh : shifts) push(ev[0], P3{ev[1] + sh.x, ev[2] + sh.y, ev[3] + sh.z});
            }
            return out;
        }
        // parallelepiped_lattice.rs:217-294: mirrors across the six faces
        const double eps = 2.220446049250313e-16;
        P3 axes[3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        P3 nrm[3];
        for (int k = 0; k < 3; ++k) {
            double nk = norm3(e[k]);
            nrm[k] = nk > eps ? P3{e[k].x / nk, e[k].y / nk, e[k].z / nk} : axes[k];
        }
        P3 pmax[3] = {P3{o.x + e[0].x, o.y + e[0].y, o.z + e[0].z}, P3{o.x + e[1].x, o.y + e[1].y, o.z + e[1].z},
                      P3{o.x + e[2].x, o.y + e[2].y, o.z + e[2].z}};
        out.reserve(n * 24);
        for (size_t q = 0; q < n; ++q) {
            const double* ev = interior + 4 * q;
            P3 p{ev[1], ev[2], ev[3]};
            for (int k = 0; k < 3; ++k) {
                P3 nn = neg3(nrm[k]);
                double d = dot3(sub3(p, o), nn);
                push(ev[0], sub3(p, scale3(nn, 2.0 * d)));
                double d2 = dot3(sub3(p, pmax[k]), nrm[k]);
                push(ev[0], sub3(p, scale3(nrm[k], 2.0 * d2)));
            }
        }
        return out;
    }
    if (kind == BGWX_LATTICE_SPHERICAL) {
        if (bc != BGWX_BC_REFLECTION) return out;  // no periodic images for a sphere
        // spherical_lattice.rs:72-131
        P3 c{params[0], params[1], params[2]};
        double radius = params[3];
        const double eps = 2.220446049250313e-16;
        out.reserve(n * 8);
        for (size_t q = 0; q < n; ++q) {
            const double* ev = interior + 4 * q;
            P3 p{ev[1], ev[2], ev[3]};
            P3 v = sub3(p, c);
            double d = norm3(v);
            if (d < eps) {
                push(ev[0], P3{c.x + radius, c.y, c.z});
                push(ev[0], P3{c.x - radius, c.y, c.z});
                continue;
            }
            P3 u{v.x / d, v.y / d, v.z / d};
            P3 q1{c.x + radius * u.x, c.y + radius * u.y, c.z + radius * u.z};
            P3 q2{c.x - radius * u.x, c.y - radius * u.y, c.z - radius * u.z};
            P3 n1 = u, n2 = neg3(u);
            P3 pq1 = sub3(p, q1);
            double dot1 = pq1.x * n1.x + pq1.y * n1.y + pq1.z * n1.z;
            push(ev[0], P3{p.x - 2.0 * dot1 * n1.x, p.y - 2.0 * dot1 * n1.y, p.z - 2.0 * dot1 * n1.z});
            P3 pq2 = sub3(p, q2);
            double dot2 = pq2.x * n2.x + pq2.y * n2.y + pq2.z * n2.z;
            push(ev[0], P3{p.x - 2.0 * dot2 * n2.x, p.y - 2.0 * dot2 * n2.y, p.z - 2.0 * dot2 * n2.z});
        }
        return out;
    }
    return out;
}

namespace {
// spacetime.rs:593-600 with nalgebra's left-to-right U4 dot.
inline double interval(const double* b, const double* a) {
    double d0 = b[0] - a[0], d1 = b[1] - a[1], d2 = b[2] - a[2], d3 = b[3] - a[3];
    return (((-d0) * d0 + d1 * d1) + d2 * d2) + d3 * d3;
}
}  // namespace

// lattice_bubbles.rs:71-119 (interior-interior, then interior-exterior).
void check_causality(const double* interior, size_t n_int, const double* exterior, size_t n_ext) {
    for (size_t a = 0; a < n_int; ++a)
        for (size_t b = a + 1; b < n_int; ++b)
            if (interval(interior + 4 * b, interior + 4 * a) < 0.0)
                throw Error{"Bubble Interior(" + std::to_string(a) + ") is formed inside bubble Interior(" +
                            std::to_string(b) + ") at initial time (overlapping light cones)"};
    for (size_t a = 0; a < n_int; ++a)
        for (size_t e = 0; e < n_ext; ++e)
            if (interval(exterior + 4 * e, interior + 4 * a) < 0.0)
                throw Error{"Bubble Interior(" + std::to_string(a) + ") is formed inside bubble Exterior(" +
                            std::to_string(e) + ") at initial time (overlapping light cones)"};
}

}  // namespace bgw
