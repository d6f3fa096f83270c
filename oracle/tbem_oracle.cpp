// CPU oracle for the dense Burton-Miller TBEM path -- TEST INFRASTRUCTURE ONLY.
//
// A plain C++ restatement of the reference (sonium-bem, Rust) CPU algorithms, used as the
// checker for the CUDA product and as the timed CPU baseline. It is compiled with
// -ffp-contract=off so that, like the Rust code it restates, no multiply-add is fused.
// Each routine cites the reference file:line it follows (paths relative to the sonium
// workspace root).

#include "tbem_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using cd = std::complex<double>;
constexpr double kPi = 3.14159265358979323846264338327950288;

// ---------------------------------------------------------------------------------------------
// Quadrature rules
// ---------------------------------------------------------------------------------------------

// Gauss-Legendre nodes/weights on [-1, 1] by Newton iteration on the three-term Legendre
// recurrence (crates/sonium-bem/src/core/integration/gauss.rs:38-84 uses the same method for the
// orders without a checked-in table; the tables of the other orders agree to rounding).
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    const int half = (n + 1) / 2;
    const double nf = static_cast<double>(n);
    for (int i = 0; i < half; ++i) {
        double root = std::cos(kPi * (i + 0.75) / (nf + 0.5));
        for (int it = 0; it < 32; ++it) {
            double p0 = 1.0, p1 = root;
            for (int d = 2; d <= n; ++d) {
                double p2 = ((2 * d - 1) * root * p1 - (d - 1) * p0) / d;
                p0 = p1;
                p1 = p2;
            }
            double dp = nf * (root * p1 - p0) / (root * root - 1.0);
            double next = root - p1 / dp;
            bool done = std::fabs(next - root) <= 4.0 * 2.220446049250313e-16 * std::max(std::fabs(next), 1.0);
            root = next;
            if (done) break;
        }
        double p0 = 1.0, p1 = root;
        for (int d = 2; d <= n; ++d) {
            double p2 = ((2 * d - 1) * root * p1 - (d - 1) * p0) / d;
            p0 = p1;
            p1 = p2;
        }
        double dp = nf * (root * p1 - p0) / (root * root - 1.0);
        double wt = 2.0 / ((1.0 - root * root) * dp * dp);
        if (n == 1) {
            root = 0.0;
            wt = 2.0;
        }
        x[i] = -root;
        x[n - 1 - i] = root;
        w[i] = wt;
        w[n - 1 - i] = wt;
    }
}

// Published symmetric triangle rules on the unit simplex (weights sum to 1): centroid rule,
// the 4-point degree-3 rule, the 7-point degree-5 rule and the 13-point degree-7 rule, with the
// same 15-digit constants the reference tables carry (gauss.rs:503-540), so that the regular
// quadrature reproduces the reference to rounding.
const double kTR1[1][3] = {{0.333333333333333, 0.333333333333333, 1.0}};
const double kTR4[4][3] = {{0.333333333333333, 0.333333333333333, -0.5625},
                           {0.6, 0.2, 0.520833333333333},
                           {0.2, 0.6, 0.520833333333333},
                           {0.2, 0.2, 0.520833333333333}};
const double kTR7[7][3] = {{0.333333333333333, 0.333333333333333, 0.225},
                           {0.797426985353087, 0.101286507323456, 0.125939180544827},
                           {0.101286507323456, 0.797426985353087, 0.125939180544827},
                           {0.101286507323456, 0.101286507323456, 0.125939180544827},
                           {0.470142064105115, 0.059715871789770, 0.132394152788506},
                           {0.059715871789770, 0.470142064105115, 0.132394152788506},
                           {0.470142064105115, 0.470142064105115, 0.132394152788506}};
const double kTR13[13][3] = {{0.333333333333333, 0.333333333333333, -0.149570044467682},
                             {0.260345966079040, 0.260345966079040, 0.175615257433208},
                             {0.260345966079040, 0.479308067841920, 0.175615257433208},
                             {0.479308067841920, 0.260345966079040, 0.175615257433208},
                             {0.065130102902216, 0.065130102902216, 0.053347235608838},
                             {0.065130102902216, 0.869739794195568, 0.053347235608838},
                             {0.869739794195568, 0.065130102902216, 0.053347235608838},
                             {0.638444188569810, 0.048690315425316, 0.077113760890257},
                             {0.048690315425316, 0.638444188569810, 0.077113760890257},
                             {0.638444188569810, 0.312865496004874, 0.077113760890257},
                             {0.312865496004874, 0.638444188569810, 0.077113760890257},
                             {0.048690315425316, 0.312865496004874, 0.077113760890257},
                             {0.312865496004874, 0.048690315425316, 0.077113760890257}};

struct TriPoint {
    double xi, eta, w;
};

// triangle_quadrature (gauss.rs:110-156): orders 1..4 are the tables above scaled to the
// reference-triangle area 0.5; higher orders are the Duffy-collapsed Gauss-Legendre product.
std::vector<TriPoint> triangle_quadrature(int order) {
    std::vector<TriPoint> out;
    auto table = [&](const double (*t)[3], int n) {
        for (int i = 0; i < n; ++i) out.push_back({t[i][0], t[i][1], t[i][2] * 0.5});
    };
    switch (order) {
        case 1: table(kTR1, 1); break;
        case 2: table(kTR4, 4); break;
        case 3: table(kTR7, 7); break;
        case 4: table(kTR13, 13); break;
        default: {
            std::vector<double> x, w;
            gauss_legendre(order, x, w);
            for (int a = 0; a < order; ++a) {
                double u = 0.5 * (x[a] + 1.0);
                double uw = 0.5 * w[a];
                for (int b = 0; b < order; ++b) {
                    double v = 0.5 * (x[b] + 1.0);
                    double vw = 0.5 * w[b];
                    out.push_back({u, (1.0 - u) * v, uw * vw * (1.0 - u)});
                }
            }
        }
    }
    return out;
}

// ---------------------------------------------------------------------------------------------
// Element geometry helpers
// ---------------------------------------------------------------------------------------------

struct Coords {
    double v[3][3];  // v[node][xyz]
};

// compute_parameters (crates/sonium-bem/src/core/integration/regular.rs:636-714), Tri3 branch.
void tri_parameters(const Coords& c, double s, double t, double pos[3], double& jac,
                    double nrm[3]) {
    const double sf[3] = {1.0 - s - t, s, t};
    const double sds[3] = {-1.0, 1.0, 0.0};
    const double sdt[3] = {-1.0, 0.0, 1.0};
    double dxs[3] = {0, 0, 0}, dxt[3] = {0, 0, 0};
    pos[0] = pos[1] = pos[2] = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            pos[j] += sf[i] * c.v[i][j];
            dxs[j] += sds[i] * c.v[i][j];
            dxt[j] += sdt[i] * c.v[i][j];
        }
    double n0 = dxs[1] * dxt[2] - dxs[2] * dxt[1];
    double n1 = dxs[2] * dxt[0] - dxs[0] * dxt[2];
    double n2 = dxs[0] * dxt[1] - dxs[1] * dxt[0];
    jac = std::sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    if (jac > 1e-15) {
        nrm[0] = n0 / jac;
        nrm[1] = n1 / jac;
        nrm[2] = n2 / jac;
    } else {
        nrm[0] = nrm[1] = nrm[2] = 0.0;
    }
}

// normalize (crates/sonium-bem/src/core/mesh/element.rs:304-311).
double normalize3(const double d[3], double u[3]) {
    double len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (len > 1e-15) {
        u[0] = d[0] / len;
        u[1] = d[1] / len;
        u[2] = d[2] / len;
        return len;
    }
    u[0] = u[1] = u[2] = 0.0;
    return 0.0;
}

inline cd exp_i(double x) { return cd(std::cos(x), std::sin(x)); }

// ---------------------------------------------------------------------------------------------
// Adaptive subdivision
// ---------------------------------------------------------------------------------------------

struct Leaf {
    double tv[3][2];
    double factor;
    int order;
};

// compute_gauss_order and the three error estimators (singular.rs:1543-1573).
int compute_gauss_order(double disfac) {
    const int gmin = 4, gmax = 7;
    const double acc = 0.0005;
    for (int o = gmin; o <= gmax; ++o) {
        double base = disfac / (2.0 * o + 1.0);
        double eg = std::pow(base, 2 * o + 1);
        double eh = std::pow(base, 2 * o + 2);
        double ee = std::pow(base, 2 * o + 3);
        if (eg < acc && eh < acc && ee < acc) return o;
    }
    return gmax;
}

// generate_subelements (singular.rs:1372-1540), Tri3 branch: breadth-first 4-way split of the
// reference triangle while dist(centre, x)/sqrt(area at level) < 3; at most 15 splits per level
// (the 16th ends the level), at most 110 leaves.
std::vector<Leaf> generate_subelements(const double x[3], const Coords& c, double area) {
    const int kMaxNse = 60, kNse = 4, kMaxLeaves = 110;
    const double kTolF = 3.0;
    static const double csi6[6] = {0.0, 1.0, 0.0, 0.5, 0.5, 0.0};
    static const double eta6[6] = {0.0, 0.0, 1.0, 0.0, 0.5, 0.5};
    std::vector<Leaf> out;
    double xs[kMaxNse][3], es[kMaxNse][3];
    for (int j = 0; j < 3; ++j) {
        xs[0][j] = csi6[j];
        es[0][j] = eta6[j];
    }
    int nsfl = 1;
    double faclin = 2.0;
    for (;;) {
        int ndie = 0;
        faclin *= 0.5;
        const double arels = area * faclin * faclin;
        const int nsel = nsfl;
        double xp[kMaxNse][3], ep[kMaxNse][3];
        std::memcpy(xp, xs, sizeof(double) * 3 * nsel);
        std::memcpy(ep, es, sizeof(double) * 3 * nsel);
        for (int idi = 0; idi < nsel; ++idi) {
            double sc = ((0.0 + xp[idi][0]) + xp[idi][1] + xp[idi][2]) / 3.0;
            double tc = ((0.0 + ep[idi][0]) + ep[idi][1] + ep[idi][2]) / 3.0;
            const double sf[3] = {1.0 - sc - tc, sc, tc};
            double g[3] = {0, 0, 0};
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) g[j] += sf[i] * c.v[i][j];
            double dx = g[0] - x[0], dy = g[1] - x[1], dz = g[2] - x[2];
            double dist = std::sqrt(dx * dx + dy * dy + dz * dz);
            double ratdis = dist / std::sqrt(arels);
            if (ratdis < kTolF) {
                ++ndie;
                if (ndie > 15) break;
                nsfl = ndie * kNse;
                const int nsf0 = nsfl - kNse;
                double xsp[6], esp[6];
                for (int j = 0; j < 3; ++j) {
                    int j1 = (j + 1) % 3;
                    xsp[j] = xp[idi][j];
                    xsp[j + 3] = (xp[idi][j] + xp[idi][j1]) / 2.0;
                    esp[j] = ep[idi][j];
                    esp[j + 3] = (ep[idi][j] + ep[idi][j1]) / 2.0;
                }
                for (int j = 0; j < 3; ++j) {
                    int nsu = nsf0 + j;
                    int j1 = j + 3;
                    int j2 = (j == 0) ? 5 : j - 1 + 3;
                    xs[nsu][0] = xsp[j];
                    xs[nsu][1] = xsp[j1];
                    xs[nsu][2] = xsp[j2];
                    es[nsu][0] = esp[j];
                    es[nsu][1] = esp[j1];
                    es[nsu][2] = esp[j2];
                }
                xs[nsf0 + 3][0] = xsp[3];
                xs[nsf0 + 3][1] = xsp[4];
                xs[nsf0 + 3][2] = xsp[5];
                es[nsf0 + 3][0] = esp[3];
                es[nsf0 + 3][1] = esp[4];
                es[nsf0 + 3][2] = esp[5];
            } else {
                Leaf lf;
                for (int j = 0; j < 3; ++j) {
                    lf.tv[j][0] = xp[idi][j];
                    lf.tv[j][1] = ep[idi][j];
                }
                lf.factor = faclin;
                lf.order = compute_gauss_order(0.5 / ratdis);
                out.push_back(lf);
                if (static_cast<int>(out.size()) >= kMaxLeaves) return out;
            }
        }
        if (ndie == 0) break;
    }
    return out;
}

struct Channels {
    cd g{0, 0}, h{0, 0}, ht{0, 0}, e{0, 0};
};

// regular_integration_with_normals_mode (regular.rs:124-321), flat normals, no derivative.
Channels regular_pair(const double x[3], const double nx[3], const Coords& c, double area,
                      const or_physics& ph) {
    const double wavruim = ph.harmonic_factor * ph.wave_number;
    const double k2 = ph.wave_number * ph.wave_number;
    Channels r;
    std::vector<Leaf> leaves = generate_subelements(x, c, area);
    for (const Leaf& lf : leaves) {
        const bool iforie = std::fabs(std::fabs(lf.factor) - 1.0) < 1e-10;
        std::vector<TriPoint> pts = triangle_quadrature(lf.order);
        for (const TriPoint& p : pts) {
            double xio, eto, weih2;
            if (iforie) {
                xio = p.xi;
                eto = p.eta;
                weih2 = p.w;
            } else {
                double l0 = 1.0 - p.xi - p.eta;
                xio = lf.tv[0][0] * l0 + lf.tv[1][0] * p.xi + lf.tv[2][0] * p.eta;
                eto = lf.tv[0][1] * l0 + lf.tv[1][1] * p.xi + lf.tv[2][1] * p.eta;
                double dx1 = lf.tv[1][0] - lf.tv[0][0];
                double dy1 = lf.tv[1][1] - lf.tv[0][1];
                double dx2 = lf.tv[2][0] - lf.tv[0][0];
                double dy2 = lf.tv[2][1] - lf.tv[0][1];
                double det = std::fabs(dx1 * dy2 - dx2 * dy1);
                weih2 = p.w * det;
            }
            double pos[3], jac, ny[3];
            tri_parameters(c, xio, eto, pos, jac, ny);
            double wga = weih2 * jac;
            double d[3] = {pos[0] - x[0], pos[1] - x[1], pos[2] - x[2]};
            double u[3];
            double dis = normalize3(d, u);
            if (dis < 1e-15) continue;
            double re1 = wavruim * dis;
            double re2 = wga / (4.0 * kPi * dis);
            cd zg = exp_i(re1) * re2;
            cd z1(-1.0 / dis, wavruim);
            cd zb = zg * z1;
            double rny = u[0] * ny[0] + u[1] * ny[1] + u[2] * ny[2];
            double rnx = -(u[0] * nx[0] + u[1] * nx[1] + u[2] * nx[2]);
            double rq = rny * rnx;
            double nxny = nx[0] * ny[0] + nx[1] * ny[1] + nx[2] * ny[2];
            double dq = dis * dis;
            cd ef((3.0 / dq - k2) * rq + nxny / dq, -wavruim / dis * (3.0 * rq + nxny));
            r.g += zg;
            r.h += zb * rny;
            r.ht += zb * rnx;
            r.e += zg * ef;
        }
    }
    return r;
}

// QuadratureParams::for_ka (singular.rs:51-85) keyed by estimate_element_size (singular.rs:1615-1640).
struct SingularParams {
    int edge_order, sub_order, sections, subtri;
};
SingularParams singular_params(const Coords& c, double k) {
    double v1[3], v2[3];
    for (int j = 0; j < 3; ++j) {
        v1[j] = c.v[1][j] - c.v[0][j];
        v2[j] = c.v[2][j] - c.v[0][j];
    }
    double cr0 = v1[1] * v2[2] - v1[2] * v2[1];
    double cr1 = v1[2] * v2[0] - v1[0] * v2[2];
    double cr2 = v1[0] * v2[1] - v1[1] * v2[0];
    double area = 0.5 * std::sqrt(cr0 * cr0 + cr1 * cr1 + cr2 * cr2);
    double size = std::max(std::sqrt(area), 1e-10);
    double ka = k * size;
    if (ka < 0.3) return {3, 4, 4, 2};
    if (ka < 1.0) return {4, 5, 6, 2};
    if (ka < 2.0) return {5, 6, 8, 3};
    return {6, 7, 10, 4};
}

// singular_integration_with_params_mode (singular.rs:297-614), Tri3, flat normals: regularised
// edge line integral for E, Duffy-collapsed sub-triangles (centroid, vertex, edge midpoint) for
// G, H, H^T and the k^2 (n_x.n_y) G part of E.
Channels singular_pair(const double x[3], const double nx[3], const Coords& c,
                       const or_physics& ph) {
    static const double csi6[6] = {0.0, 1.0, 0.0, 0.5, 0.5, 0.0};
    static const double eta6[6] = {0.0, 0.0, 1.0, 0.0, 0.5, 0.5};
    const double wavruim = ph.harmonic_factor * ph.wave_number;
    const double k2 = ph.wave_number * ph.wave_number;
    const SingularParams q = singular_params(c, ph.wave_number);
    std::vector<double> ecx, ecw, scx, scw;
    gauss_legendre(q.edge_order, ecx, ecw);
    gauss_legendre(q.sub_order, scx, scw);
    const int nsec1 = q.sections, nsec2 = q.subtri;
    Channels r;
    for (int ieg = 0; ieg < 3; ++ieg) {
        const int ig1 = (ieg + 1) % 3, ig2 = ieg + 3;
        double dp[3];
        double leneg = 0.0;
        for (int i = 0; i < 3; ++i) {
            dp[i] = c.v[ig1][i] - c.v[ieg][i];
            leneg += dp[i] * dp[i];
        }
        leneg = std::sqrt(leneg);
        const double dpo[3] = {dp[0] / leneg, dp[1] / leneg, dp[2] / leneg};
        const double leneg_scaled = leneg / (2.0 * nsec1);
        cd zre(0, 0);
        const double delsec = 2.0 / nsec1;
        double secmid = -1.0 - delsec / 2.0;
        for (int is = 0; is < nsec1; ++is) {
            secmid += delsec;
            for (int ig = 0; ig < q.edge_order; ++ig) {
                double sga = secmid + ecx[ig] / nsec1;
                double wga = ecw[ig] * leneg_scaled;
                double d[3];
                for (int i = 0; i < 3; ++i) {
                    double gp = c.v[ieg][i] + dp[i] * (sga + 1.0) / 2.0;
                    d[i] = gp - x[i];
                }
                double u[3];
                double dis = normalize3(d, u);
                if (dis < 1e-15) continue;
                double re1 = wavruim * dis;
                double re2 = 4.0 * kPi * dis;
                cd zg = exp_i(re1) / re2;
                cd z1(-1.0 / dis, wavruim);
                cd zf = zg * z1;
                cd zd[3] = {zf * u[0], zf * u[1], zf * u[2]};
                cd w0 = zd[1] * dpo[2] - zd[2] * dpo[1];
                cd w1 = zd[2] * dpo[0] - zd[0] * dpo[2];
                cd w2 = zd[0] * dpo[1] - zd[1] * dpo[0];
                zre += (w0 * nx[0] + w1 * nx[1] + w2 * nx[2]) * wga;
            }
        }
        r.e += zre;
        for (int isec = 0; isec < nsec2; ++isec) {
            const double aresub = 1.0 / 24.0 / nsec2;
            double ss[3], ts[3];
            ss[0] = 1.0 / 3.0;
            ts[0] = 1.0 / 3.0;
            if (isec == 0) {
                ss[1] = csi6[ieg];
                ss[2] = csi6[ig2];
                ts[1] = eta6[ieg];
                ts[2] = eta6[ig2];
            } else {
                ss[1] = csi6[ig2];
                ss[2] = csi6[ig1];
                ts[1] = eta6[ig2];
                ts[2] = eta6[ig1];
            }
            for (int a = 0; a < q.sub_order; ++a) {
                const double sga = scx[a];
                for (int b = 0; b < q.sub_order; ++b) {
                    const double tga = scx[b];
                    const double wei = scw[a] * scw[b];
                    double sgg = 0.5 * (1.0 - sga) * ss[0] +
                                 0.25 * (1.0 + sga) * ((1.0 - tga) * ss[1] + (1.0 + tga) * ss[2]);
                    double tgg = 0.5 * (1.0 - sga) * ts[0] +
                                 0.25 * (1.0 + sga) * ((1.0 - tga) * ts[1] + (1.0 + tga) * ts[2]);
                    double pos[3], jac, ny[3];
                    tri_parameters(c, sgg, tgg, pos, jac, ny);
                    double wga = wei * (1.0 + sga) * aresub * jac;
                    double d[3] = {pos[0] - x[0], pos[1] - x[1], pos[2] - x[2]};
                    double u[3];
                    double dis = normalize3(d, u);
                    if (dis < 1e-15) continue;
                    double re1 = wavruim * dis;
                    double re2 = wga / (4.0 * kPi * dis);
                    cd zg = exp_i(re1) * re2;
                    cd z1(-1.0 / dis, wavruim);
                    cd zb = zg * z1;
                    double rny = u[0] * ny[0] + u[1] * ny[1] + u[2] * ny[2];
                    double rnx = -(u[0] * nx[0] + u[1] * nx[1] + u[2] * nx[2]);
                    r.g += zg;
                    r.h += zb * rny;
                    r.ht += zb * rnx;
                    double nd = nx[0] * ny[0] + nx[1] * ny[1] + nx[2] * ny[2];
                    r.e += zg * k2 * nd;
                }
            }
        }
    }
    return r;
}

struct ElementGeom {
    std::vector<double> center, normal, area;
};

// compute_element_geometry (generators.rs:771-830), Tri3.
void element_geometry(int64_t m, const double* nodes, const uint32_t* tris, double* centers,
                      double* normals, double* areas) {
    for (int64_t e = 0; e < m; ++e) {
        const uint32_t* t = tris + 3 * e;
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int a = 0; a < 3; ++a) s += nodes[3 * t[a] + j];
            centers[3 * e + j] = s / 3.0;
        }
        double v1[3], v2[3];
        for (int j = 0; j < 3; ++j) {
            v1[j] = nodes[3 * t[1] + j] - nodes[3 * t[0] + j];
            v2[j] = nodes[3 * t[2] + j] - nodes[3 * t[0] + j];
        }
        double cr[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2],
                        v1[0] * v2[1] - v1[1] * v2[0]};
        double len = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        areas[e] = len / 2.0;
        if (len > 1e-15) {
            normals[3 * e + 0] = cr[0] / len;
            normals[3 * e + 1] = cr[1] / len;
            normals[3 * e + 2] = cr[2] / len;
        } else {
            normals[3 * e + 0] = normals[3 * e + 1] = normals[3 * e + 2] = 0.0;
        }
    }
}

inline cd C(const or_c128& v) { return cd(v.re, v.im); }
inline or_c128 O(const cd& v) { return or_c128{v.real(), v.imag()}; }

struct BcView {
    int kind;
    cd value;
    bool has_adm;
    cd adm;
};
BcView bc_at(const or_bc* bc, int64_t e) {
    BcView v{0, cd(0, 0), false, cd(0, 0)};
    if (!bc) return v;
    if (bc->kind) v.kind = bc->kind[e];
    if (bc->value) v.value = C(bc->value[e]);
    if (bc->has_adm && bc->has_adm[e]) {
        v.has_adm = true;
        if (bc->adm) v.adm = C(bc->adm[e]);
    }
    return v;
}

void set_threads(int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
}

// build_tbem_system_with_beta_parallel (tbem.rs:1284-1466) for rows [row0, row1): free terms
// and the per-field-BC coefficients over the channels that `channels(i, j, x, nx)` returns (the
// CPU integration rules, or channels computed elsewhere for the same pairs).
template <class ChannelFn>
int assemble_rows_impl(int64_t n_nodes, const double* nodes, int64_t m, const uint32_t* tris, const or_bc* bc,
                       const or_physics* ph, or_c128 beta_in, int64_t row0, int64_t row1, int threads,
                       or_c128* A, or_c128* rhs, ChannelFn&& channels) {
    if (m <= 0 || row0 < 0 || row1 > m || row0 > row1) return 1;
    for (int64_t i = 0; i < 3 * m; ++i)
        if (tris[i] >= static_cast<uint64_t>(n_nodes)) return 1;
    std::vector<double> centers(3 * m), normals(3 * m), areas(m);
    element_geometry(m, nodes, tris, centers.data(), normals.data(), areas.data());
    const cd gamma(1.0, 0.0), tau(ph->tau, 0.0), iwr(0.0, ph->pressure_factor);
    const cd beta = C(beta_in);
    std::vector<BcView> bcs(m);
    for (int64_t e = 0; e < m; ++e) bcs[e] = bc_at(bc, e);
    const int64_t rows = row1 - row0;
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t rr = 0; rr < rows; ++rr) {
        const int64_t i = row0 + rr;
        or_c128* row = A + rr * m;
        std::vector<cd> local(m, cd(0, 0));
        cd lrhs(0, 0);
        const BcView& sb = bcs[i];
        // Free terms (tbem.rs:1344-1358).
        if (sb.kind == 0) {
            local[i] -= gamma * 0.5;
            if (sb.has_adm) local[i] -= sb.adm * iwr * beta * tau * 0.5;
            lrhs += sb.value * iwr * beta * tau * 0.5;
        } else if (sb.kind == 1) {
            local[i] += beta * tau * 0.5;
            lrhs -= sb.value * gamma * 0.5;
        }
        const double* x = &centers[3 * i];
        const double* nx = &normals[3 * i];
        for (int64_t j = 0; j < m; ++j) {
            const BcView& fb = bcs[j];
            const bool compute_rhs = std::abs(fb.value) > 1e-15;
            const Channels r = channels(i, j, x, nx, areas[j]);
            // Coefficient per field BC (tbem.rs:1404-1417).
            cd coeff(0, 0);
            if (fb.kind == 0) {
                coeff = r.h * gamma * tau + r.e * beta;
                if (fb.has_adm) coeff -= (r.g * gamma * tau + r.ht * beta) * fb.adm * iwr;
            } else if (fb.kind == 1) {
                coeff = -(r.g * gamma * tau + r.ht * beta);
            }
            local[j] += coeff;
            if (compute_rhs) {
                if (fb.kind == 0)
                    lrhs += (r.g * gamma * tau + r.ht * beta) * fb.value * iwr;
                else if (fb.kind == 1)
                    lrhs += (r.h * gamma * tau + r.e * beta) * fb.value;
            }
        }
        for (int64_t j = 0; j < m; ++j) row[j] = O(local[j]);
        if (rhs) rhs[rr] = O(lrhs);
    }
    return 0;
}

std::vector<Coords> element_coords(int64_t m, const double* nodes, const uint32_t* tris) {
    std::vector<Coords> coords(m);
    for (int64_t e = 0; e < m; ++e)
        for (int a = 0; a < 3; ++a)
            for (int j = 0; j < 3; ++j) coords[e].v[a][j] = nodes[3 * tris[3 * e + a] + j];
    return coords;
}

// ---------------------------------------------------------------------------------------------
// Quadrature charts of the reference CUDA assembly path: the records that its chart-driven pair
// kernel (sonium_bem_quadrature_pair_c64, crates/sonium-compute/src/cuda/kernels/bem_kernels.cu:
// 839-967) integrates. The record layouts are the kernel's (bem_kernels.cu:818-833), so that the
// reference kernel, compiled from its own source, can be run on them as a checker.
// ---------------------------------------------------------------------------------------------
static_assert(sizeof(or_chart_sample) == 96, "SoniumBemQuadratureSampleC64 layout");
static_assert(sizeof(or_chart_pair) == 64, "SoniumBemQuadraturePairC64 layout");

// append_regular_tri3_quadrature (tbem.rs:4998-5049): every leaf of generate_subelements, its
// triangle rule mapped affinely by the leaf's vertices (weight times the map's determinant), the
// point's position, Jacobian and normal from the element map; kind 0 (full channels).
void chart_regular(const double x[3], const Coords& c, double area, std::vector<or_chart_sample>& out) {
    for (const Leaf& lf : generate_subelements(x, c, area)) {
        for (const TriPoint& p : triangle_quadrature(lf.order)) {
            const double l0 = 1.0 - p.xi - p.eta;
            const double mxi = lf.tv[0][0] * l0 + lf.tv[1][0] * p.xi + lf.tv[2][0] * p.eta;
            const double meta = lf.tv[0][1] * l0 + lf.tv[1][1] * p.xi + lf.tv[2][1] * p.eta;
            const double dx1 = lf.tv[1][0] - lf.tv[0][0], dy1 = lf.tv[1][1] - lf.tv[0][1];
            const double dx2 = lf.tv[2][0] - lf.tv[0][0], dy2 = lf.tv[2][1] - lf.tv[0][1];
            const double det = std::fabs(dx1 * dy2 - dx2 * dy1);
            or_chart_sample smp{};
            double jac;
            tri_parameters(c, mxi, meta, smp.position, jac, smp.field_normal);
            smp.weight = p.w * det * jac;
            smp.basis_weight = 1.0;
            smp.kind = 0;
            out.push_back(smp);
        }
    }
}

// append_singular_tri3_quadrature(_with_params) (tbem.rs:5051-5161): the regularised edge line
// integral (kind 2: position on the edge, unit edge direction, weight = GL weight times the
// section's half length) and the Duffy-collapsed bulk of the sub-triangles (kind 1), with the rule
// of QuadratureParams::for_ka at ka = k sqrt(area).
void chart_singular(const Coords& c, double area, double k, std::vector<or_chart_sample>& out) {
    static const double csi6[6] = {0.0, 1.0, 0.0, 0.5, 0.5, 0.0};
    static const double eta6[6] = {0.0, 0.0, 1.0, 0.0, 0.5, 0.5};
    const double ka = k * std::max(std::sqrt(area), 1e-10);
    SingularParams q;
    if (ka < 0.3) q = {3, 4, 4, 2};
    else if (ka < 1.0) q = {4, 5, 6, 2};
    else if (ka < 2.0) q = {5, 6, 8, 3};
    else q = {6, 7, 10, 4};
    std::vector<double> ex, ew, sx, sw;
    gauss_legendre(q.edge_order, ex, ew);
    gauss_legendre(q.sub_order, sx, sw);
    for (int edge = 0; edge < 3; ++edge) {
        const int next = (edge + 1) % 3;
        double d[3];
        for (int j = 0; j < 3; ++j) d[j] = c.v[next][j] - c.v[edge][j];
        const double len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        const double scale = len / (2.0 * q.sections);
        for (int sec = 0; sec < q.sections; ++sec) {
            const double mid = -1.0 + (sec + 0.5) * (2.0 / q.sections);
            for (int g = 0; g < q.edge_order; ++g) {
                const double loc = mid + ex[g] / q.sections;
                or_chart_sample smp{};
                for (int j = 0; j < 3; ++j) {
                    smp.position[j] = c.v[edge][j] + d[j] * (loc + 1.0) / 2.0;
                    smp.edge_direction[j] = d[j] / len;
                }
                smp.weight = ew[g] * scale;
                smp.basis_weight = 1.0;
                smp.kind = 2;
                out.push_back(smp);
            }
        }
    }
    for (int edge = 0; edge < 3; ++edge) {
        const int next = (edge + 1) % 3, ig2 = edge + 3;
        for (int st = 0; st < q.subtri; ++st) {
            const double area_scale = 1.0 / 24.0 / q.subtri;
            const double ss[3] = {1.0 / 3.0, st == 0 ? csi6[edge] : csi6[ig2], st == 0 ? csi6[ig2] : csi6[next]};
            const double ts[3] = {1.0 / 3.0, st == 0 ? eta6[edge] : eta6[ig2], st == 0 ? eta6[ig2] : eta6[next]};
            for (int a = 0; a < q.sub_order; ++a) {
                const double sga = sx[a];
                for (int b = 0; b < q.sub_order; ++b) {
                    const double tga = sx[b];
                    const double xi = 0.5 * (1.0 - sga) * ss[0] +
                                      0.25 * (1.0 + sga) * ((1.0 - tga) * ss[1] + (1.0 + tga) * ss[2]);
                    const double eta = 0.5 * (1.0 - sga) * ts[0] +
                                       0.25 * (1.0 + sga) * ((1.0 - tga) * ts[1] + (1.0 + tga) * ts[2]);
                    or_chart_sample smp{};
                    double jac;
                    tri_parameters(c, xi, eta, smp.position, jac, smp.field_normal);
                    smp.weight = sw[a] * sw[b] * (1.0 + sga) * area_scale * jac;
                    smp.basis_weight = 1.0;
                    smp.kind = 1;
                    out.push_back(smp);
                }
            }
        }
    }
}

}  // namespace

extern "C" {

// PhysicsParams::new_with_convention (types.rs:165-190) with the shared e^{-i omega t}
// convention (spatial sign +1, crates/sonium-bem/src/core/conventions.rs:308-313).
void or_physics_new(double frequency, double c, double rho, int is_internal, or_physics* out) {
    const double omega = 2.0 * kPi * frequency;
    out->frequency = frequency;
    out->speed_of_sound = c;
    out->density = rho;
    out->omega = omega;
    out->wave_number = omega / c;
    out->wave_length = c / frequency;
    out->harmonic_factor = 1.0;
    out->pressure_factor = rho * omega * 1.0;
    out->tau = is_internal ? -1.0 : 1.0;
}

int or_icosphere_counts(int level, int64_t* n_nodes, int64_t* n_tris) {
    if (level < 0 || level > 9) return 1;
    int64_t f = 20;
    for (int i = 0; i < level; ++i) f *= 4;
    *n_tris = f;
    *n_nodes = f / 2 + 2;
    return 0;
}

// generate_icosphere_mesh (generators.rs:309-397) and get_midpoint (generators.rs:400-428).
// The 12 icosahedron vertices and 20 faces are the standard golden-ratio construction; the
// face order and the (v0, m01, m20), (v1, m12, m01), (v2, m20, m12), (m01, m12, m20) split
// order follow the reference so that element numbering matches.
int or_icosphere(double radius, int level, double sx, double sy, double sz, double* nodes,
                 uint32_t* tris) {
    int64_t nn, nt;
    if (or_icosphere_counts(level, &nn, &nt)) return 1;
    const double phi = (1.0 + std::sqrt(5.0)) / 2.0;
    std::vector<std::array<double, 3>> v = {
        {-1.0, phi, 0.0}, {1.0, phi, 0.0},  {-1.0, -phi, 0.0}, {1.0, -phi, 0.0},
        {0.0, -1.0, phi}, {0.0, 1.0, phi},  {0.0, -1.0, -phi}, {0.0, 1.0, -phi},
        {phi, 0.0, -1.0}, {phi, 0.0, 1.0},  {-phi, 0.0, -1.0}, {-phi, 0.0, 1.0}};
    for (auto& p : v) {
        double len = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        p[0] /= len;
        p[1] /= len;
        p[2] /= len;
    }
    std::vector<std::array<uint32_t, 3>> f = {
        {0, 11, 5}, {0, 5, 1},  {0, 1, 7},   {0, 7, 10}, {0, 10, 11}, {1, 5, 9},  {5, 11, 4},
        {11, 10, 2}, {10, 7, 6}, {7, 1, 8},  {3, 9, 4},  {3, 4, 2},   {3, 2, 6},  {3, 6, 8},
        {3, 8, 9},  {4, 9, 5},  {2, 4, 11},  {6, 2, 10}, {8, 6, 7},   {9, 8, 1}};
    for (int l = 0; l < level; ++l) {
        std::vector<std::array<uint32_t, 3>> nf;
        nf.reserve(f.size() * 4);
        // Edge-midpoint cache keyed by the ordered vertex pair (dense map per level).
        std::vector<std::vector<std::pair<uint32_t, uint32_t>>> cache(v.size());
        auto mid = [&](uint32_t a, uint32_t b) -> uint32_t {
            uint32_t lo = std::min(a, b), hi = std::max(a, b);
            for (auto& kv : cache[lo])
                if (kv.first == hi) return kv.second;
            std::array<double, 3> m = {(v[a][0] + v[b][0]) / 2.0, (v[a][1] + v[b][1]) / 2.0,
                                       (v[a][2] + v[b][2]) / 2.0};
            double len = std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
            m = {m[0] / len, m[1] / len, m[2] / len};
            uint32_t idx = static_cast<uint32_t>(v.size());
            v.push_back(m);
            cache[lo].push_back({hi, idx});
            return idx;
        };
        for (auto& t : f) {
            uint32_t m01 = mid(t[0], t[1]);
            uint32_t m12 = mid(t[1], t[2]);
            uint32_t m20 = mid(t[2], t[0]);
            nf.push_back({t[0], m01, m20});
            nf.push_back({t[1], m12, m01});
            nf.push_back({t[2], m20, m12});
            nf.push_back({m01, m12, m20});
        }
        f.swap(nf);
    }
    if (static_cast<int64_t>(v.size()) != nn || static_cast<int64_t>(f.size()) != nt) return 2;
    for (size_t i = 0; i < v.size(); ++i) {
        nodes[3 * i + 0] = v[i][0] * radius * sx;
        nodes[3 * i + 1] = v[i][1] * radius * sy;
        nodes[3 * i + 2] = v[i][2] * radius * sz;
    }
    for (size_t i = 0; i < f.size(); ++i)
        for (int j = 0; j < 3; ++j) tris[3 * i + j] = f[i][j];
    return 0;
}

void or_element_geometry(int64_t n_tris, const double* nodes, const uint32_t* tris,
                         double* centers, double* normals, double* areas) {
    element_geometry(n_tris, nodes, tris, centers, normals, areas);
}

int or_assemble_rows(int64_t n_nodes, const double* nodes, int64_t m, const uint32_t* tris,
                     const or_bc* bc, const or_physics* ph, or_c128 beta_in, int64_t row0,
                     int64_t row1, int threads, or_c128* A, or_c128* rhs) {
    if (m <= 0) return 1;
    for (int64_t i = 0; i < 3 * m; ++i)
        if (tris[i] >= static_cast<uint64_t>(n_nodes)) return 1;
    const std::vector<Coords> coords = element_coords(m, nodes, tris);
    return assemble_rows_impl(n_nodes, nodes, m, tris, bc, ph, beta_in, row0, row1, threads, A, rhs,
                              [&](int64_t i, int64_t j, const double* x, const double* nx, double area) {
                                  return (j == i) ? singular_pair(x, nx, coords[j], *ph)
                                                  : regular_pair(x, nx, coords[j], area, *ph);
                              });
}

int or_assemble_rows_from_channels(int64_t n_nodes, const double* nodes, int64_t m, const uint32_t* tris,
                                   const or_bc* bc, const or_physics* ph, or_c128 beta, int64_t row0,
                                   int64_t row1, const or_c128* channels, int threads, or_c128* A, or_c128* rhs) {
    if (!channels) return 1;
    return assemble_rows_impl(n_nodes, nodes, m, tris, bc, ph, beta, row0, row1, threads, A, rhs,
                              [&](int64_t i, int64_t j, const double*, const double*, double) {
                                  const or_c128* c4 = channels + ((i - row0) * m + j) * 4;
                                  Channels r;
                                  r.g = C(c4[0]);
                                  r.h = C(c4[1]);
                                  r.ht = C(c4[2]);
                                  r.e = C(c4[3]);
                                  return r;
                              });
}

int64_t or_chart_rows(int64_t n_nodes, const double* nodes, int64_t m, const uint32_t* tris, double k,
                      int64_t row0, int64_t row1, int threads, or_chart_pair* pairs, or_chart_sample* samples,
                      int64_t capacity) {
    if (m <= 0 || row0 < 0 || row1 > m || row0 > row1) return -1;
    for (int64_t i = 0; i < 3 * m; ++i)
        if (tris[i] >= static_cast<uint64_t>(n_nodes)) return -1;
    const std::vector<Coords> coords = element_coords(m, nodes, tris);
    std::vector<double> centers(3 * m), normals(3 * m), areas(m);
    element_geometry(m, nodes, tris, centers.data(), normals.data(), areas.data());
    const int64_t rows = row1 - row0;
    std::vector<std::vector<or_chart_sample>> per_row(rows);
    std::vector<std::vector<int64_t>> counts(rows);
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t rr = 0; rr < rows; ++rr) {
        const int64_t i = row0 + rr;
        auto& out = per_row[rr];
        counts[rr].resize(m);
        for (int64_t j = 0; j < m; ++j) {
            const size_t before = out.size();
            if (j == i)
                chart_singular(coords[j], areas[j], k, out);
            else
                chart_regular(&centers[3 * i], coords[j], areas[j], out);
            counts[rr][j] = static_cast<int64_t>(out.size() - before);
        }
    }
    int64_t total = 0;
    for (const auto& v : per_row) total += static_cast<int64_t>(v.size());
    if (!pairs || !samples) return total;
    if (capacity < total) return -1;
    int64_t off = 0;
    for (int64_t rr = 0; rr < rows; ++rr) {
        const int64_t i = row0 + rr;
        for (int64_t j = 0; j < m; ++j) {
            or_chart_pair& p = pairs[rr * m + j];
            for (int d = 0; d < 3; ++d) {
                p.source_point[d] = centers[3 * i + d];
                p.source_normal[d] = normals[3 * i + d];
            }
            p.sample_offset = static_cast<uint64_t>(off);
            p.sample_count = static_cast<uint64_t>(counts[rr][j]);
            off += counts[rr][j];
        }
        std::memcpy(samples + (off - static_cast<int64_t>(per_row[rr].size())), per_row[rr].data(),
                    per_row[rr].size() * sizeof(or_chart_sample));
    }
    return total;
}

void or_regular_pair(const double* x, const double* nx, const double* c9, double area,
                     const or_physics* ph, or_c128* out4) {
    Coords c;
    std::memcpy(c.v, c9, sizeof(c.v));
    Channels r = regular_pair(x, nx, c, area, *ph);
    out4[0] = O(r.g);
    out4[1] = O(r.h);
    out4[2] = O(r.ht);
    out4[3] = O(r.e);
}

void or_singular_pair(const double* x, const double* nx, const double* c9, const or_physics* ph,
                      or_c128* out4) {
    Coords c;
    std::memcpy(c.v, c9, sizeof(c.v));
    Channels r = singular_pair(x, nx, c, *ph);
    out4[0] = O(r.g);
    out4[1] = O(r.h);
    out4[2] = O(r.ht);
    out4[3] = O(r.e);
}

int or_subelements(const double* x, const double* c9, double area, double* leaves, int cap) {
    Coords c;
    std::memcpy(c.v, c9, sizeof(c.v));
    std::vector<Leaf> l = generate_subelements(x, c, area);
    for (int i = 0; i < static_cast<int>(l.size()) && i < cap; ++i) {
        double* o = leaves + 8 * i;
        for (int a = 0; a < 3; ++a) {
            o[2 * a] = l[i].tv[a][0];
            o[2 * a + 1] = l[i].tv[a][1];
        }
        o[6] = l[i].factor;
        o[7] = l[i].order;
    }
    return static_cast<int>(l.size());
}

void or_rhs_plane_wave(int64_t n, const double* centers, const double* normals,
                       const or_physics* ph, or_c128 beta_in, int64_t r, const double* dirs,
                       const or_c128* amps, or_c128* rhs) {
    const double k = ph->wave_number, s = ph->harmonic_factor;
    const cd gamma(1.0, 0.0), tau(ph->tau, 0.0), beta = C(beta_in);
    for (int64_t i = 0; i < n; ++i) {
        const double* p = centers + 3 * i;
        const double* nn = normals + 3 * i;
        for (int64_t q = 0; q < r; ++q) {
            const double* d = dirs + 3 * q;
            const cd a = amps ? C(amps[q]) : cd(1.0, 0.0);
            double kdotx = s * k * (d[0] * p[0] + d[1] * p[1] + d[2] * p[2]);
            cd pinc = a * exp_i(kdotx);
            double kdotn = s * k * (d[0] * nn[0] + d[1] * nn[1] + d[2] * nn[2]);
            cd dpdn = cd(0.0, kdotn) * (a * exp_i(kdotx));
            rhs[i * r + q] = O(-(gamma * pinc + beta * tau * dpdn));
        }
    }
}

void or_matvec(int64_t n, const or_c128* A, const or_c128* x, or_c128* y, int threads) {
    set_threads(threads);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        cd s(0, 0);
        const or_c128* row = A + i * n;
        for (int64_t j = 0; j < n; ++j) s += C(row[j]) * C(x[j]);
        y[i] = O(s);
    }
}

}  // extern "C"

namespace {

// ---------------------------------------------------------------------------------------------
// GMRES (gmres.rs:631-1047; givens_rotation / solve_upper_triangular gmres_common.rs:91-127)
// ---------------------------------------------------------------------------------------------

struct DenseOp {
    int64_t n;
    const or_c128* A;
    long matvecs = 0;
    void apply(const std::vector<cd>& x, std::vector<cd>& y) {
        ++matvecs;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            cd s(0, 0);
            const or_c128* row = A + i * n;
            for (int64_t j = 0; j < n; ++j) s += C(row[j]) * x[j];
            y[i] = s;
        }
    }
};

double vnorm(const std::vector<cd>& v) {
    double s = 0.0;
    for (const cd& z : v) s += std::norm(z);
    return std::sqrt(s);
}

cd dotc(const cd* a, const std::vector<cd>& b, int64_t n) {
    cd s(0, 0);
    for (int64_t i = 0; i < n; ++i) s += std::conj(a[i]) * b[i];
    return s;
}

void givens(cd a, cd b, cd& c, cd& s) {
    const double tol = 1e-30;
    if (std::abs(b) < tol) {
        c = 1.0;
        s = 0.0;
        return;
    }
    if (std::abs(a) < tol) {
        c = 0.0;
        s = 1.0;
        return;
    }
    double r = std::sqrt(std::norm(a) + std::norm(b));
    c = a * (1.0 / r);
    s = b * (1.0 / r);
}

std::vector<cd> upper_solve(const std::vector<cd>& h, int64_t ld, const std::vector<cd>& g,
                            int64_t k) {
    std::vector<cd> y(k, cd(0, 0));
    for (int64_t i = k - 1; i >= 0; --i) {
        cd s = g[i];
        for (int64_t j = i + 1; j < k; ++j) s -= h[i * ld + j] * y[j];
        if (std::abs(h[i * ld + i]) > 1e-30) y[i] = s * (1.0 / h[i * ld + i]);
    }
    return y;
}

}  // namespace

extern "C" int or_gmres(int64_t n, const or_c128* A, const or_c128* b_in, const or_c128* x0,
                        int64_t max_it, int64_t restart, double tol, int threads, or_c128* x_out,
                        or_gmres_result* res) {
    set_threads(threads);
    std::memset(res, 0, sizeof(*res));
    std::vector<cd> b(n), x(n, cd(0, 0)), op(n), w(n);
    for (int64_t i = 0; i < n; ++i) b[i] = C(b_in[i]);
    if (x0)
        for (int64_t i = 0; i < n; ++i) x[i] = C(x0[i]);
    auto write_out = [&]() {
        for (int64_t i = 0; i < n; ++i) x_out[i] = O(x[i]);
    };
    if (max_it <= 0 || restart <= 0 || !(tol > 0.0) || !std::isfinite(tol)) {
        res->status = 3;
        write_out();
        return 1;
    }
    DenseOp A_op{n, A};
    const int64_t m = restart;
    const double bn_raw = vnorm(b);
    const bool rhs_zero = bn_raw < 1e-15;
    const double bnorm = rhs_zero ? 1.0 : bn_raw;
    const double pbnorm = bnorm;  // identity preconditioner
    std::vector<cd> V((m + 1) * n);
    std::vector<cd> H((m + 1) * m);
    std::vector<cd> cs, sn, g(m + 1), coeffs, rco;
    int64_t total = 0, restarts = 0;
    int status = 1;
    bool converged = false;
    double est = 1.0, resid = 1.0;
    auto true_rel = [&]() {
        A_op.apply(x, op);
        double s = 0;
        for (int64_t k = 0; k < n; ++k) s += std::norm(b[k] - op[k]);
        return std::sqrt(s) / bnorm;
    };
    for (int64_t outer = 0; outer < max_it && !converged && status == 1; ++outer) {
        A_op.apply(x, op);
        for (int64_t k = 0; k < n; ++k) op[k] = b[k] - op[k];
        double trel = vnorm(op) / bnorm;
        w = op;
        double beta = vnorm(w);
        double rel = beta / pbnorm;
        if (rel < tol && trel < tol) {
            converged = true;
            status = 0;
            est = rel;
            resid = trel;
            break;
        }
        if (!std::isfinite(beta) || beta == 0.0) {
            status = 2;
            est = rel;
            resid = trel;
            break;
        }
        const double ib = 1.0 / beta;
        for (int64_t k = 0; k < n; ++k) V[k] = w[k] * ib;
        std::fill(H.begin(), H.end(), cd(0, 0));
        cs.clear();
        sn.clear();
        std::fill(g.begin(), g.end(), cd(0, 0));
        g[0] = beta;
        bool restart_now = false;
        for (int64_t j = 0; j < m; ++j) {
            ++total;
            A_op.apply(std::vector<cd>(V.begin() + j * n, V.begin() + (j + 1) * n), w);
            const double wnb = vnorm(w);
            coeffs.assign(j + 1, cd(0, 0));
            for (int64_t i = 0; i <= j; ++i) coeffs[i] = dotc(&V[i * n], w, n);
            for (int64_t i = 0; i <= j; ++i) H[i * m + j] = coeffs[i];
            for (int64_t i = 0; i <= j; ++i)
                for (int64_t k = 0; k < n; ++k) w[k] -= coeffs[i] * V[i * n + k];
            double wn = vnorm(w);
            if (wn < 0.707 * wnb) {
                rco.assign(j + 1, cd(0, 0));
                for (int64_t i = 0; i <= j; ++i) rco[i] = dotc(&V[i * n], w, n);
                for (int64_t i = 0; i <= j; ++i) H[i * m + j] += rco[i];
                for (int64_t i = 0; i <= j; ++i)
                    for (int64_t k = 0; k < n; ++k) w[k] -= rco[i] * V[i * n + k];
                wn = vnorm(w);
            }
            H[(j + 1) * m + j] = wn;
            bool inner_conv = false;
            if (wn < 1e-20) {
                inner_conv = true;
            } else {
                const double inv = 1.0 / wn;
                for (int64_t k = 0; k < n; ++k) V[(j + 1) * n + k] = w[k] * inv;
            }
            for (int64_t i = 0; i < j; ++i) {
                cd t = std::conj(cs[i]) * H[i * m + j] + std::conj(sn[i]) * H[(i + 1) * m + j];
                H[(i + 1) * m + j] = cd(0, 0) - sn[i] * H[i * m + j] + cs[i] * H[(i + 1) * m + j];
                H[i * m + j] = t;
            }
            cd c, s;
            givens(H[j * m + j], H[(j + 1) * m + j], c, s);
            cs.push_back(c);
            sn.push_back(s);
            H[j * m + j] = std::conj(c) * H[j * m + j] + std::conj(s) * H[(j + 1) * m + j];
            H[(j + 1) * m + j] = 0.0;
            cd t = std::conj(c) * g[j] + std::conj(s) * g[j + 1];
            g[j + 1] = cd(0, 0) - s * g[j] + c * g[j + 1];
            g[j] = t;
            const double absr = std::abs(g[j + 1]);
            const double relr = absr / pbnorm;
            const bool conv = relr < tol || (!inner_conv && absr < 1e-20);
            if (conv) {
                std::vector<cd> y = upper_solve(H, m, g, j + 1);
                for (int64_t i = 0; i <= j; ++i)
                    for (int64_t k = 0; k < n; ++k) x[k] += y[i] * V[i * n + k];
                double tr = true_rel();
                if (tr >= tol && tr >= 1e-20) {
                    ++restarts;
                    restart_now = true;
                    break;
                }
                converged = true;
                status = 0;
                est = relr;
                resid = tr;
                break;
            }
            if (inner_conv) {
                std::vector<cd> y = upper_solve(H, m, g, j + 1);
                for (int64_t i = 0; i <= j; ++i)
                    for (int64_t k = 0; k < n; ++k) x[k] += y[i] * V[i * n + k];
                double ar = true_rel();
                est = relr;
                resid = ar;
                if (ar < tol) {
                    converged = true;
                    status = 0;
                } else {
                    status = 2;
                }
                break;
            }
        }
        if (converged || status != 1) break;
        if (restart_now) continue;
        std::vector<cd> y = upper_solve(H, m, g, m);
        for (int64_t i = 0; i < m; ++i)
            for (int64_t k = 0; k < n; ++k) x[k] += y[i] * V[i * n + k];
        double tr = true_rel();
        if (tr < tol) {
            converged = true;
            status = 0;
            est = tr;
            resid = tr;
            break;
        }
        ++restarts;
    }
    if (!converged && status == 1) {
        resid = true_rel();
        est = resid;
    }
    // finalize_gmres_solution (gmres.rs:159-247): one more product for the published residual.
    A_op.apply(x, op);
    double rs = 0, axs = 0, bs = 0;
    for (int64_t k = 0; k < n; ++k) {
        rs += std::norm(b[k] - op[k]);
        axs += std::norm(op[k]);
        bs += std::norm(b[k]);
    }
    const double rn = std::sqrt(rs), bn = std::sqrt(bs);
    res->residual = bn > 0 ? rn / bn : rn;
    res->backward_error = rn / std::max(std::sqrt(axs) + bn, 2.2250738585072014e-308);
    res->estimated_residual = est;
    (void)resid;
    res->iterations = total;
    res->restarts = restarts;
    res->matvecs = A_op.matvecs;
    res->converged = converged ? 1 : 0;
    res->status = status;
    write_out();
    return 0;
}

// ---------------------------------------------------------------------------------------------
// Mie series (crates/sonium-wave/src/analytical/solutions_3d.rs:315-366, 769-900)
// ---------------------------------------------------------------------------------------------

extern "C" double or_sph_j(int n, double x) {
    if (std::fabs(x) < 1e-10) return n == 0 ? 1.0 : 0.0;
    if (std::fabs(x) < 1e-4) {
        double x2 = x * x;
        if (n == 0) return 1.0 - x2 / 6.0 + x2 * x2 / 120.0;
        if (n == 1) return x * (1.0 / 3.0 - x2 / 30.0 + x2 * x2 / 840.0);
    }
    if (n == 0) return std::sin(x) / x;
    if (n == 1) return std::sin(x) / (x * x) - std::cos(x) / x;
    // Miller's downward recurrence j_{k} = (2k+3)/x j_{k+1} - j_{k+2}, normalised by j0 or j1.
    const int start = n + static_cast<int>(std::fabs(x)) + 20;
    std::vector<double> val(start + 1, 0.0);
    double jn1 = 0.0, jc = 1e-30;
    val[start] = jc;
    for (int k = start - 1; k >= 0; --k) {
        double jp = (2 * k + 3) / x * jc - jn1;
        val[k] = jp;
        jn1 = jc;
        jc = jp;
    }
    double j0 = std::sin(x) / x;
    double j1 = std::sin(x) / (x * x) - std::cos(x) / x;
    double scale = std::fabs(j0) >= std::fabs(j1) ? j0 / val[0] : j1 / val[1];
    return val[n] * scale;
}

extern "C" double or_sph_y(int n, double x) {
    if (std::fabs(x) < 1e-10) return -INFINITY;
    double y0 = -std::cos(x) / x;
    if (n == 0) return y0;
    double y1 = -std::cos(x) / (x * x) - std::sin(x) / x;
    if (n == 1) return y1;
    // Upward recurrence y_{k} = (2k-1)/x y_{k-1} - y_{k-2}.
    double a = y0, b = y1;
    for (int k = 2; k <= n; ++k) {
        double c = (2 * k - 1) / x * b - a;
        a = b;
        b = c;
    }
    return b;
}

extern "C" void or_mie_rigid_coefficients(double ka, int nt, or_c128* out) {
    for (int n = 0; n < nt; ++n) {
        double jn = or_sph_j(n, ka), yn = or_sph_y(n, ka);
        double jm = n > 0 ? or_sph_j(n - 1, ka) : std::cos(ka) / ka;
        double ym = n > 0 ? or_sph_y(n - 1, ka) : std::sin(ka) / ka;
        double jp = jm - (n + 1.0) / ka * jn;
        double yp = ym - (n + 1.0) / ka * yn;
        cd a = cd(jp, 0.0) / cd(jp, yp);
        out[n] = O(a);
    }
}

extern "C" void or_mie_rigid_field(double k, double radius, int nt, double r, int64_t nth,
                                   const double* theta, or_c128* out) {
    std::vector<or_c128> co(nt);
    or_mie_rigid_coefficients(k * radius, nt, co.data());
    const double kr = k * r;
    std::vector<double> jn(nt), yn(nt);
    for (int n = 0; n < nt; ++n) {
        jn[n] = or_sph_j(n, kr);
        yn[n] = or_sph_y(n, kr);
    }
    for (int64_t t = 0; t < nth; ++t) {
        const double ct = std::cos(theta[t]);
        cd tot(0, 0);
        double p0 = 1.0, p1 = ct;
        for (int n = 0; n < nt; ++n) {
            double pn;
            if (n == 0)
                pn = 1.0;
            else if (n == 1)
                pn = ct;
            else {
                pn = ((2.0 * n - 1.0) * ct * p1 - (n - 1.0) * p0) / n;
                p0 = p1;
                p1 = pn;
            }
            cd ipn(std::cos(n * kPi / 2.0), std::sin(n * kPi / 2.0));
            cd hn(jn[n], yn[n]);
            tot += (2.0 * n + 1.0) * ipn * (jn[n] - C(co[n]) * hn) * pn;
        }
        out[t] = O(tot);
    }
}

// ---------------------------------------------------------------------------------------------
// Exterior field evaluation, constant Tri3 surface data
// ---------------------------------------------------------------------------------------------
// compute_scattered_field_with_incident (crates/sonium-bem/src/core/postprocess/pressure.rs:
// 1388-1448) with explicit surface velocity (constant_cauchy_data, :1489-1491) ->
// integrate_element_field (:1566-1606, Tri3: the 7-point rule of triangle_quadrature(3)) ->
// integrate_quad_point (:1987-2042), geometry by quadrature_geometry (element.rs:420-464).
// p_scat(x) = sum_e sum_q [ p_e dG/dn_y - v_e (i pressure_factor) G ] J w_q.
extern "C" void or_field_eval(const double* nodes, const uint32_t* tris, int64_t n_tris,
                              const or_c128* pressure, const or_c128* velocity, double k,
                              double harmonic_factor, double pressure_factor, const double* points,
                              int64_t m, int threads, or_c128* out) {
    const std::vector<TriPoint> rule = triangle_quadrature(3);
    const double wavruim = k * harmonic_factor;
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t i = 0; i < m; ++i) {
        const double* x = points + 3 * i;
        cd acc(0.0, 0.0);
        for (int64_t e = 0; e < n_tris; ++e) {
            Coords c;
            for (int a = 0; a < 3; ++a)
                for (int d = 0; d < 3; ++d) c.v[a][d] = nodes[3 * (int64_t)tris[3 * e + a] + d];
            const cd p_surf = C(pressure[e]);
            const cd v_surf = velocity ? C(velocity[e]) : cd(0.0, 0.0);
            cd contrib_e(0.0, 0.0);
            for (const TriPoint& q : rule) {
                double pos[3], jac, nrm[3];
                tri_parameters(c, q.xi, q.eta, pos, jac, nrm);
                if (jac < 1e-15) continue;
                const double rv[3] = {pos[0] - x[0], pos[1] - x[1], pos[2] - x[2]};
                const double r = std::sqrt(rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2]);
                if (r < 1e-15) continue;
                const double vjacwe = jac * q.w;
                const cd zgrfu = exp_i(wavruim * r) / (4.0 * kPi * r);
                const cd zgikr = zgrfu * cd(-1.0 / r, wavruim);
                const double drdn = (rv[0] * nrm[0] + rv[1] * nrm[1] + rv[2] * nrm[2]) / r;
                cd contrib = p_surf * (zgikr * drdn) * vjacwe;
                if (std::abs(v_surf) > 1e-15) contrib -= v_surf * cd(0.0, pressure_factor) * zgrfu * vjacwe;
                contrib_e += contrib;
            }
            acc += contrib_e;
        }
        out[i] = O(acc);
    }
}

// =============================================================================================
// Discontinuous Tri3 bases: build_tbem_system_linear (crates/sonium-bem/src/core/assembly/
// tbem.rs:1490-1620) and build_tbem_system_discontinuous_stabilized (:2810-2990) with
// regular_integration_linear_with_normals (integration/regular.rs:359-470) and
// singular_integration_linear_with_params_mode (integration/singular.rs:868-1170). NB = 3
// (linear) or 6 (quadratic) DOFs per element, collocated at the interior points of
// mesh/element.rs:91-115, basis_values of element.rs:229-262; element e owns DOFs NB e + c.
// =============================================================================================
namespace {

const double kLinColl[3][2] = {{1.0 / 6.0, 1.0 / 6.0}, {2.0 / 3.0, 1.0 / 6.0}, {1.0 / 6.0, 2.0 / 3.0}};
const double kQuadColl[6][2] = {{0.0915762135097715, 0.0915762135097715}, {0.8168475729804585, 0.0915762135097715},
                                {0.0915762135097715, 0.8168475729804585}, {0.445948490915965, 0.445948490915965},
                                {0.445948490915965, 0.108103018168070},   {0.108103018168070, 0.445948490915965}};

inline void coll_local(int nb, int q, double& s, double& t) {
    s = nb == 6 ? kQuadColl[q][0] : kLinColl[q][0];
    t = nb == 6 ? kQuadColl[q][1] : kLinColl[q][1];
}

// basis_values (element.rs:229-262), Tri3: linear 2 lambda - 1/3, quadratic Lagrange.
inline void panel_basis(int nbas, double s, double t, double nb[6]) {
    const double l[3] = {1.0 - s - t, s, t};
    if (nbas == 3) {
        for (int b = 0; b < 3; ++b) nb[b] = 2.0 * l[b] - 1.0 / 3.0;
        return;
    }
    nb[0] = l[0] * (2.0 * l[0] - 1.0);
    nb[1] = l[1] * (2.0 * l[1] - 1.0);
    nb[2] = l[2] * (2.0 * l[2] - 1.0);
    nb[3] = 4.0 * l[0] * l[1];
    nb[4] = 4.0 * l[1] * l[2];
    nb[5] = 4.0 * l[2] * l[0];
}

// Reference derivatives of the basis (panel_basis_gradients, singular.rs:1180-1195).
inline void panel_deriv(int nbas, double s, double t, double d[6][2]) {
    if (nbas == 3) {
        const double dd[3][2] = {{-2.0, -2.0}, {2.0, 0.0}, {0.0, 2.0}};
        std::memcpy(d, dd, sizeof(dd));
        return;
    }
    const double l = 1.0 - s - t;
    const double dd[6][2] = {{1.0 - 4.0 * l, 1.0 - 4.0 * l}, {4.0 * s - 1.0, 0.0}, {0.0, 4.0 * t - 1.0},
                             {4.0 * (l - s), -4.0 * s},      {4.0 * t, 4.0 * s},   {-4.0 * t, 4.0 * (l - t)}};
    std::memcpy(d, dd, sizeof(dd));
}

// local_to_global (element.rs:65-76), Tri3 shape functions.
void lin_point(const Coords& c, double s, double t, double x[3]) {
    const double sf[3] = {1.0 - s - t, s, t};
    x[0] = x[1] = x[2] = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) x[j] += sf[i] * c.v[i][j];
}

struct Channels3 {
    Channels b[6];
};

// regular_integration_linear_with_normals (regular.rs:359-470), flat normals.
Channels3 regular_pair_linear(const double x[3], const double nx[3], const Coords& c, double area,
                              const or_physics& ph, int nbas = 3) {
    const double wavruim = ph.harmonic_factor * ph.wave_number;
    const double k2 = ph.wave_number * ph.wave_number;
    Channels3 r;
    std::vector<Leaf> leaves = generate_subelements(x, c, area);
    for (const Leaf& lf : leaves) {
        const bool iforie = std::fabs(std::fabs(lf.factor) - 1.0) < 1e-10;
        std::vector<TriPoint> pts = triangle_quadrature(lf.order);
        for (const TriPoint& p : pts) {
            double xio, eto, weih2;
            if (iforie) {
                xio = p.xi;
                eto = p.eta;
                weih2 = p.w;
            } else {
                double l0 = 1.0 - p.xi - p.eta;
                xio = lf.tv[0][0] * l0 + lf.tv[1][0] * p.xi + lf.tv[2][0] * p.eta;
                eto = lf.tv[0][1] * l0 + lf.tv[1][1] * p.xi + lf.tv[2][1] * p.eta;
                double dx1 = lf.tv[1][0] - lf.tv[0][0];
                double dy1 = lf.tv[1][1] - lf.tv[0][1];
                double dx2 = lf.tv[2][0] - lf.tv[0][0];
                double dy2 = lf.tv[2][1] - lf.tv[0][1];
                weih2 = p.w * std::fabs(dx1 * dy2 - dx2 * dy1);
            }
            double pos[3], jac, ny[3];
            tri_parameters(c, xio, eto, pos, jac, ny);
            double wga = weih2 * jac;
            double d[3] = {pos[0] - x[0], pos[1] - x[1], pos[2] - x[2]};
            double u[3];
            double dis = normalize3(d, u);
            if (dis < 1e-15) continue;
            cd zg = exp_i(wavruim * dis) * (wga / (4.0 * kPi * dis));
            cd zb = zg * cd(-1.0 / dis, wavruim);
            double rny = u[0] * ny[0] + u[1] * ny[1] + u[2] * ny[2];
            double rnx = -(u[0] * nx[0] + u[1] * nx[1] + u[2] * nx[2]);
            double rq = rny * rnx;
            double nxny = nx[0] * ny[0] + nx[1] * ny[1] + nx[2] * ny[2];
            double dq = dis * dis;
            cd ef((3.0 / dq - k2) * rq + nxny / dq, -wavruim / dis * (3.0 * rq + nxny));
            cd zh = zb * rny, zt = zb * rnx, ze = zg * ef;
            double nb[6];
            panel_basis(nbas, xio, eto, nb);
            for (int b = 0; b < nbas; ++b) {
                r.b[b].g += zg * nb[b];
                r.b[b].h += zh * nb[b];
                r.b[b].ht += zt * nb[b];
                r.b[b].e += ze * nb[b];
            }
        }
    }
    return r;
}

// panel_basis_gradients (singular.rs:1173-1258), Tri3: surface gradients of the basis functions
// at (s, t) from the panel's tangents and metric.
void lin_gradients(const Coords& c, int nbas, double s, double t, double grad[6][3]) {
    double der[6][2];
    panel_deriv(nbas, s, t, der);
    const double sds[3] = {-1.0, 1.0, 0.0}, sdt[3] = {-1.0, 0.0, 1.0};
    double ts[3] = {0, 0, 0}, tt[3] = {0, 0, 0};
    for (int node = 0; node < 3; ++node)
        for (int a = 0; a < 3; ++a) {
            ts[a] += sds[node] * c.v[node][a];
            tt[a] += sdt[node] * c.v[node][a];
        }
    double ss = 0, tq = 0, st = 0;
    for (int a = 0; a < 3; ++a) {
        ss += ts[a] * ts[a];
        tq += tt[a] * tt[a];
        st += ts[a] * tt[a];
    }
    const double det = ss * tq - st * st;
    for (int b = 0; b < nbas; ++b) {
        const double ga = (tq * der[b][0] - st * der[b][1]) / det;
        const double gb = (ss * der[b][1] - st * der[b][0]) / det;
        for (int a = 0; a < 3; ++a) grad[b][a] = ga * ts[a] + gb * tt[a];
    }
}

// singular_integration_linear_with_params_mode (singular.rs:868-1170), Tri3, flat normals, no
// derivative: the edge line integral of the regularised E weighted by the basis at the edge
// point, the centroid-centred Duffy sub-triangles for G, H, H^T and the area part of E
// (k^2 n_x.n_y G N_b plus the basis-gradient term of the weighted Stokes identity).
Channels3 singular_pair_linear(const double x[3], const double nx[3], const Coords& c,
                               const or_physics& ph, int nbas = 3) {
    static const double csi6[6] = {0.0, 1.0, 0.0, 0.5, 0.5, 0.0};
    static const double eta6[6] = {0.0, 0.0, 1.0, 0.0, 0.5, 0.5};
    const double wavruim = ph.harmonic_factor * ph.wave_number;
    const double k2 = ph.wave_number * ph.wave_number;
    const SingularParams q = singular_params(c, ph.wave_number);
    std::vector<double> ecx, ecw, scx, scw;
    gauss_legendre(q.edge_order, ecx, ecw);
    gauss_legendre(q.sub_order, scx, scw);
    const int nsec1 = q.sections, nsec2 = q.subtri;
    Channels3 r;
    for (int ieg = 0; ieg < 3; ++ieg) {
        const int ig1 = (ieg + 1) % 3, ig2 = ieg + 3;
        double dp[3];
        double leneg = 0.0;
        for (int i = 0; i < 3; ++i) {
            dp[i] = c.v[ig1][i] - c.v[ieg][i];
            leneg += dp[i] * dp[i];
        }
        leneg = std::sqrt(leneg);
        const double dpo[3] = {dp[0] / leneg, dp[1] / leneg, dp[2] / leneg};
        const double leneg_scaled = leneg / (2.0 * nsec1);
        const double delsec = 2.0 / nsec1;
        double secmid = -1.0 - delsec / 2.0;
        for (int is = 0; is < nsec1; ++is) {
            secmid += delsec;
            for (int ig = 0; ig < q.edge_order; ++ig) {
                double sga = secmid + ecx[ig] / nsec1;
                double wga = ecw[ig] * leneg_scaled;
                double d[3];
                for (int i = 0; i < 3; ++i) {
                    double gp = c.v[ieg][i] + dp[i] * (sga + 1.0) / 2.0;
                    d[i] = gp - x[i];
                }
                double u[3];
                double dis = normalize3(d, u);
                if (dis < 1e-15) continue;
                cd zg = exp_i(wavruim * dis) / (4.0 * kPi * dis);
                cd zf = zg * cd(-1.0 / dis, wavruim);
                cd zd[3] = {zf * u[0], zf * u[1], zf * u[2]};
                cd w0 = zd[1] * dpo[2] - zd[2] * dpo[1];
                cd w1 = zd[2] * dpo[0] - zd[0] * dpo[2];
                cd w2 = zd[0] * dpo[1] - zd[1] * dpo[0];
                cd contrib = (w0 * nx[0] + w1 * nx[1] + w2 * nx[2]) * wga;
                const double te = (sga + 1.0) / 2.0;
                const double sl = csi6[ieg] * (1.0 - te) + csi6[ig1] * te;
                const double tl = eta6[ieg] * (1.0 - te) + eta6[ig1] * te;
                double nb[6];
                panel_basis(nbas, sl, tl, nb);
                for (int b = 0; b < nbas; ++b) r.b[b].e += contrib * nb[b];
            }
        }
        for (int isec = 0; isec < nsec2; ++isec) {
            const double aresub = 1.0 / 24.0 / nsec2;
            double ss[3], ts[3];
            ss[0] = 1.0 / 3.0;
            ts[0] = 1.0 / 3.0;
            if (isec == 0) {
                ss[1] = csi6[ieg];
                ss[2] = csi6[ig2];
                ts[1] = eta6[ieg];
                ts[2] = eta6[ig2];
            } else {
                ss[1] = csi6[ig2];
                ss[2] = csi6[ig1];
                ts[1] = eta6[ig2];
                ts[2] = eta6[ig1];
            }
            for (int a = 0; a < q.sub_order; ++a) {
                const double sga = scx[a];
                for (int b2 = 0; b2 < q.sub_order; ++b2) {
                    const double tga = scx[b2];
                    const double wei = scw[a] * scw[b2];
                    double sgg = 0.5 * (1.0 - sga) * ss[0] +
                                 0.25 * (1.0 + sga) * ((1.0 - tga) * ss[1] + (1.0 + tga) * ss[2]);
                    double tgg = 0.5 * (1.0 - sga) * ts[0] +
                                 0.25 * (1.0 + sga) * ((1.0 - tga) * ts[1] + (1.0 + tga) * ts[2]);
                    double pos[3], jac, ny[3];
                    tri_parameters(c, sgg, tgg, pos, jac, ny);
                    double wga = wei * (1.0 + sga) * aresub * jac;
                    double d[3] = {pos[0] - x[0], pos[1] - x[1], pos[2] - x[2]};
                    double u[3];
                    double dis = normalize3(d, u);
                    if (dis < 1e-15) continue;
                    cd zg = exp_i(wavruim * dis) * (wga / (4.0 * kPi * dis));
                    cd zb = zg * cd(-1.0 / dis, wavruim);
                    double rny = u[0] * ny[0] + u[1] * ny[1] + u[2] * ny[2];
                    double rnx = -(u[0] * nx[0] + u[1] * nx[1] + u[2] * nx[2]);
                    cd zh = zb * rny, zt = zb * rnx;
                    double nd = nx[0] * ny[0] + nx[1] * ny[1] + nx[2] * ny[2];
                    cd earea = zg * k2 * nd;
                    double nb[6], grad[6][3];
                    panel_basis(nbas, sgg, tgg, nb);
                    lin_gradients(c, nbas, sgg, tgg, grad);
                    for (int b = 0; b < nbas; ++b) {
                        r.b[b].g += zg * nb[b];
                        r.b[b].h += zh * nb[b];
                        r.b[b].ht += zt * nb[b];
                        const double gr = grad[b][0] * u[0] + grad[b][1] * u[1] + grad[b][2] * u[2];
                        const double gs = grad[b][0] * nx[0] + grad[b][1] * nx[1] + grad[b][2] * nx[2];
                        r.b[b].e += earea * nb[b] + zb * (-nd * gr + rny * gs);
                    }
                }
            }
        }
    }
    return r;
}

}  // namespace

extern "C" {

// Collocation points and normals of a discontinuous basis: nbas per element (element.rs:91-115
// through local_to_global; flat normals, tbem.rs:1516-1527).
void or_disc_collocation(int64_t n_tris, const double* nodes, const uint32_t* tris, int nbas, double* points,
                         double* normals) {
    std::vector<double> centers(3 * n_tris), nrm(3 * n_tris), areas(n_tris);
    element_geometry(n_tris, nodes, tris, centers.data(), nrm.data(), areas.data());
    for (int64_t e = 0; e < n_tris; ++e) {
        Coords c;
        for (int a = 0; a < 3; ++a)
            for (int j = 0; j < 3; ++j) c.v[a][j] = nodes[3 * tris[3 * e + a] + j];
        for (int q = 0; q < nbas; ++q) {
            double sq, tq;
            coll_local(nbas, q, sq, tq);
            lin_point(c, sq, tq, points + 3 * (nbas * e + q));
            for (int j = 0; j < 3; ++j) normals[3 * (nbas * e + q) + j] = nrm[3 * e + j];
        }
    }
}

void or_linear_collocation(int64_t n_tris, const double* nodes, const uint32_t* tris, double* points,
                           double* normals) {
    or_disc_collocation(n_tris, nodes, tris, 3, points, normals);
}

// build_tbem_system_linear (tbem.rs:1490-1620) and, with nbas 3 or 6 and sign +-1,
// build_tbem_system_discontinuous_stabilized (:2810-2990): A is (nbas m) x (nbas m) row-major.
// Prescribed boundary values are read per element (one value; the DOFs of an element share it
// through the free terms' average, tbem.rs:1248-1281, and the field BC's first basis slot).
int or_assemble_discontinuous(int64_t n_nodes, const double* nodes, int64_t m, const uint32_t* tris,
                              const or_bc* bc, const or_physics* ph, or_c128 beta_in, int nbas, double sign,
                              int threads, or_c128* A, or_c128* rhs) {
    if (m <= 0 || (nbas != 3 && nbas != 6)) return 1;
    for (int64_t i = 0; i < 3 * m; ++i)
        if (tris[i] >= static_cast<uint64_t>(n_nodes)) return 1;
    std::vector<double> centers(3 * m), normals(3 * m), areas(m);
    element_geometry(m, nodes, tris, centers.data(), normals.data(), areas.data());
    std::vector<Coords> coords(m);
    for (int64_t e = 0; e < m; ++e)
        for (int a = 0; a < 3; ++a)
            for (int j = 0; j < 3; ++j) coords[e].v[a][j] = nodes[3 * tris[3 * e + a] + j];
    const cd gamma(1.0, 0.0), tau(ph->tau, 0.0), iwr(0.0, ph->pressure_factor);
    const cd beta = C(beta_in);
    std::vector<BcView> bcs(m);
    for (int64_t e = 0; e < m; ++e) bcs[e] = bc_at(bc, e);
    const int64_t n = nbas * m;
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t r = 0; r < n; ++r) {
        const int64_t i = r / nbas;
        const int cq = static_cast<int>(r % nbas);
        std::vector<cd> local(n, cd(0, 0));
        cd lrhs(0, 0);
        const BcView& sb = bcs[i];
        if (sb.kind == 0) {  // add_free_terms (tbem.rs:1248-1281)
            local[r] -= sign * (gamma * 0.5);
            if (sb.has_adm) local[r] -= sign * sb.adm * iwr * beta * tau * 0.5;
            lrhs += sb.value * iwr * beta * tau * 0.5 * sign;
        } else if (sb.kind == 1) {
            local[r] += sign * (beta * tau * 0.5);
            lrhs -= sb.value * gamma * 0.5 * sign;
        }
        double x[3], sq, tq;
        coll_local(nbas, cq, sq, tq);
        lin_point(coords[i], sq, tq, x);
        const double* nx = &normals[3 * i];
        for (int64_t j = 0; j < m; ++j) {
            const BcView& fb = bcs[j];
            const bool compute_rhs = std::abs(fb.value) > 1e-15;
            Channels3 rr = (j == i) ? singular_pair_linear(x, nx, coords[j], *ph, nbas)
                                    : regular_pair_linear(x, nx, coords[j], areas[j], *ph, nbas);
            for (int b = 0; b < nbas; ++b) {
                const Channels& q = rr.b[b];
                cd coeff(0, 0);
                if (fb.kind == 0) {
                    coeff = sign * (q.h * gamma * tau + q.e * beta);
                    if (fb.has_adm) coeff -= sign * (q.g * gamma * tau + q.ht * beta) * fb.adm * iwr;
                } else if (fb.kind == 1) {
                    coeff = -sign * (q.g * gamma * tau + q.ht * beta);
                }
                local[nbas * j + b] += coeff;
                if (compute_rhs && b == 0) {  // values.get(b): one prescribed value per element
                    if (fb.kind == 0)
                        lrhs += (q.g * gamma * tau + q.ht * beta) * fb.value * iwr;
                    else if (fb.kind == 1)
                        lrhs += -(q.h * gamma * tau + q.e * beta) * fb.value;
                }
            }
        }
        for (int64_t j = 0; j < n; ++j) A[r * n + j] = O(local[j]);
        if (rhs) rhs[r] = O(lrhs);
    }
    return 0;
}

int or_assemble_linear(int64_t n_nodes, const double* nodes, int64_t m, const uint32_t* tris,
                       const or_bc* bc, const or_physics* ph, or_c128 beta_in, int threads, or_c128* A,
                       or_c128* rhs) {
    return or_assemble_discontinuous(n_nodes, nodes, m, tris, bc, ph, beta_in, 3, 1.0, threads, A, rhs);
}

}  // extern "C"

extern "C" {

// Pair-level access to the discontinuous-basis channels (tests): out = (g, h, ht, e) per basis.
void or_regular_pair_disc(const double* x, const double* nx, const double* c9, double area,
                          const or_physics* ph, int nbas, or_c128* out) {
    Coords c;
    std::memcpy(c.v, c9, sizeof(c.v));
    Channels3 r = regular_pair_linear(x, nx, c, area, *ph, nbas);
    for (int b = 0; b < nbas; ++b) {
        out[4 * b + 0] = O(r.b[b].g);
        out[4 * b + 1] = O(r.b[b].h);
        out[4 * b + 2] = O(r.b[b].ht);
        out[4 * b + 3] = O(r.b[b].e);
    }
}

void or_singular_pair_disc(const double* x, const double* nx, const double* c9, const or_physics* ph, int nbas,
                           or_c128* out) {
    Coords c;
    std::memcpy(c.v, c9, sizeof(c.v));
    Channels3 r = singular_pair_linear(x, nx, c, *ph, nbas);
    for (int b = 0; b < nbas; ++b) {
        out[4 * b + 0] = O(r.b[b].g);
        out[4 * b + 1] = O(r.b[b].h);
        out[4 * b + 2] = O(r.b[b].ht);
        out[4 * b + 3] = O(r.b[b].e);
    }
}

}  // extern "C"

// =============================================================================================
// Quad4 constant panels (the ElementType::Quad4 branches of the constant path): element
// geometry (compute_element_geometry, mesh/generators.rs:771-850, with compute_element_area,
// mesh/element.rs:326-362), compute_parameters (integration/regular.rs:636-714, bilinear on
// [-1, 1]^2 with vertices (1, 1), (-1, 1), (-1, -1), (1, -1)), generate_subelements
// (integration/singular.rs:1372-1540, four quads per split about the subelement centre, leaves
// mapped by centre and edge factor), quad_quadrature (integration/gauss.rs:159-170) and the
// Quad4 branch of singular_integration_with_params_mode (integration/singular.rs:297-614).
// =============================================================================================
namespace {

const double kCsi8[8] = {1.0, -1.0, -1.0, 1.0, 0.0, -1.0, 0.0, 1.0};
const double kEta8[8] = {1.0, 1.0, -1.0, -1.0, 1.0, 0.0, -1.0, 0.0};

struct Coords4 {
    double v[4][3];
};

void quad_parameters(const Coords4& c, double s, double t, double pos[3], double& jac, double nrm[3]) {
    const double s1 = 0.25 * (s + 1.0), s2 = 0.25 * (s - 1.0), t1 = t + 1.0, t2 = t - 1.0;
    const double sf[4] = {s1 * t1, -s2 * t1, s2 * t2, -s1 * t2};
    const double sds[4] = {0.25 * (t + 1.0), -0.25 * (t + 1.0), 0.25 * (t - 1.0), -0.25 * (t - 1.0)};
    const double sdt[4] = {0.25 * (s + 1.0), 0.25 * (1.0 - s), 0.25 * (s - 1.0), -0.25 * (s + 1.0)};
    double dxs[3] = {0, 0, 0}, dxt[3] = {0, 0, 0};
    pos[0] = pos[1] = pos[2] = 0.0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 3; ++j) {
            pos[j] += sf[i] * c.v[i][j];
            dxs[j] += sds[i] * c.v[i][j];
            dxt[j] += sdt[i] * c.v[i][j];
        }
    double n0 = dxs[1] * dxt[2] - dxs[2] * dxt[1];
    double n1 = dxs[2] * dxt[0] - dxs[0] * dxt[2];
    double n2 = dxs[0] * dxt[1] - dxs[1] * dxt[0];
    jac = std::sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    if (jac > 1e-15) {
        nrm[0] = n0 / jac;
        nrm[1] = n1 / jac;
        nrm[2] = n2 / jac;
    } else {
        nrm[0] = nrm[1] = nrm[2] = 0.0;
    }
}

struct QuadLeaf {
    double xc, ec, factor;
    int order;
};

std::vector<QuadLeaf> generate_subelements_quad(const double x[3], const Coords4& c, double area) {
    const int kMaxNse = 60, kNse = 4, kMaxLeaves = 110;
    std::vector<QuadLeaf> out;
    double xs[kMaxNse][4], es[kMaxNse][4];
    for (int j = 0; j < 4; ++j) {
        xs[0][j] = kCsi8[j];
        es[0][j] = kEta8[j];
    }
    int nsfl = 1;
    double faclin = 2.0;
    for (;;) {
        int ndie = 0;
        faclin *= 0.5;
        const double arels = area * faclin * faclin;
        const int nsel = nsfl;
        double xp[kMaxNse][4], ep[kMaxNse][4];
        std::memcpy(xp, xs, sizeof(double) * 4 * nsel);
        std::memcpy(ep, es, sizeof(double) * 4 * nsel);
        for (int idi = 0; idi < nsel; ++idi) {
            const double sc = (((0.0 + xp[idi][0]) + xp[idi][1]) + xp[idi][2] + xp[idi][3]) / 4.0;
            const double tc = (((0.0 + ep[idi][0]) + ep[idi][1]) + ep[idi][2] + ep[idi][3]) / 4.0;
            double g[3], jac, nrm[3];
            quad_parameters(c, sc, tc, g, jac, nrm);
            double dx = g[0] - x[0], dy = g[1] - x[1], dz = g[2] - x[2];
            double ratdis = std::sqrt(dx * dx + dy * dy + dz * dz) / std::sqrt(arels);
            if (ratdis < 3.0) {
                ++ndie;
                if (ndie > 15) break;
                nsfl = ndie * kNse;
                const int nsf0 = nsfl - kNse;
                double xsp[8], esp[8];
                for (int j = 0; j < 4; ++j) {
                    int j1 = (j + 1) % 4;
                    xsp[j] = xp[idi][j];
                    xsp[j + 4] = (xp[idi][j] + xp[idi][j1]) / 2.0;
                    esp[j] = ep[idi][j];
                    esp[j + 4] = (ep[idi][j] + ep[idi][j1]) / 2.0;
                }
                for (int j = 0; j < 4; ++j) {
                    const int nsu = nsf0 + j, j1 = j + 4, j2 = (j == 0) ? 7 : j - 1 + 4;
                    xs[nsu][0] = xsp[j];
                    xs[nsu][1] = xsp[j1];
                    xs[nsu][2] = sc;
                    xs[nsu][3] = xsp[j2];
                    es[nsu][0] = esp[j];
                    es[nsu][1] = esp[j1];
                    es[nsu][2] = tc;
                    es[nsu][3] = esp[j2];
                }
            } else {
                QuadLeaf lf;
                lf.xc = (((0.0 + xp[idi][0]) + xp[idi][1]) + xp[idi][2] + xp[idi][3]) / 4.0;
                lf.ec = (((0.0 + ep[idi][0]) + ep[idi][1]) + ep[idi][2] + ep[idi][3]) / 4.0;
                lf.factor = faclin;
                lf.order = compute_gauss_order(0.5 / ratdis);
                out.push_back(lf);
                if (static_cast<int>(out.size()) >= kMaxLeaves) return out;
            }
        }
        if (ndie == 0) break;
    }
    return out;
}

Channels regular_pair_quad(const double x[3], const double nx[3], const Coords4& c, double area,
                           const or_physics& ph) {
    const double wavruim = ph.harmonic_factor * ph.wave_number;
    const double k2 = ph.wave_number * ph.wave_number;
    Channels r;
    for (const QuadLeaf& lf : generate_subelements_quad(x, c, area)) {
        const bool iforie = std::fabs(std::fabs(lf.factor) - 1.0) < 1e-10;
        std::vector<double> gx, gw;
        gauss_legendre(lf.order, gx, gw);
        for (int a = 0; a < lf.order; ++a)
            for (int b = 0; b < lf.order; ++b) {
                const double csi = gx[a], eta = gx[b], wq = gw[a] * gw[b];
                double xio, eto, weih2;
                if (iforie) {
                    xio = csi;
                    eto = eta;
                    weih2 = wq;
                } else {
                    xio = lf.xc + csi * lf.factor;
                    eto = lf.ec + eta * lf.factor;
                    weih2 = wq * (lf.factor * lf.factor);
                }
                double pos[3], jac, ny[3];
                quad_parameters(c, xio, eto, pos, jac, ny);
                double wga = weih2 * jac;
                double d[3] = {pos[0] - x[0], pos[1] - x[1], pos[2] - x[2]};
                double u[3];
                double dis = normalize3(d, u);
                if (dis < 1e-15) continue;
                cd zg = exp_i(wavruim * dis) * (wga / (4.0 * kPi * dis));
                cd zb = zg * cd(-1.0 / dis, wavruim);
                double rny = u[0] * ny[0] + u[1] * ny[1] + u[2] * ny[2];
                double rnx = -(u[0] * nx[0] + u[1] * nx[1] + u[2] * nx[2]);
                double rq = rny * rnx;
                double nxny = nx[0] * ny[0] + nx[1] * ny[1] + nx[2] * ny[2];
                double dq = dis * dis;
                cd ef((3.0 / dq - k2) * rq + nxny / dq, -wavruim / dis * (3.0 * rq + nxny));
                r.g += zg;
                r.h += zb * rny;
                r.ht += zb * rnx;
                r.e += zg * ef;
            }
    }
    return r;
}

// estimate_element_size (singular.rs:1641-1676), Quad4: sqrt of the two triangles split on the
// diagonal 0-2.
double quad_size(const Coords4& c) {
    double v1[3], v2[3], v3[3];
    for (int j = 0; j < 3; ++j) {
        v1[j] = c.v[1][j] - c.v[0][j];
        v2[j] = c.v[2][j] - c.v[0][j];
        v3[j] = c.v[3][j] - c.v[0][j];
    }
    double c1[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2], v1[0] * v2[1] - v1[1] * v2[0]};
    double c2[3] = {v2[1] * v3[2] - v2[2] * v3[1], v2[2] * v3[0] - v2[0] * v3[2], v2[0] * v3[1] - v2[1] * v3[0]};
    double a1 = 0.5 * std::sqrt(c1[0] * c1[0] + c1[1] * c1[1] + c1[2] * c1[2]);
    double a2 = 0.5 * std::sqrt(c2[0] * c2[0] + c2[1] * c2[1] + c2[2] * c2[2]);
    return std::max(std::sqrt(a1 + a2), 1e-10);
}

Channels singular_pair_quad(const double x[3], const double nx[3], const Coords4& c, const or_physics& ph) {
    const double wavruim = ph.harmonic_factor * ph.wave_number;
    const double k2 = ph.wave_number * ph.wave_number;
    const double ka = ph.wave_number * quad_size(c);
    SingularParams q;
    if (ka < 0.3) q = {3, 4, 4, 2};
    else if (ka < 1.0) q = {4, 5, 6, 2};
    else if (ka < 2.0) q = {5, 6, 8, 3};
    else q = {6, 7, 10, 4};
    std::vector<double> ecx, ecw, scx, scw;
    gauss_legendre(q.edge_order, ecx, ecw);
    gauss_legendre(q.sub_order, scx, scw);
    const int nsec1 = q.sections, nsec2 = q.subtri;
    Channels r;
    for (int ieg = 0; ieg < 4; ++ieg) {
        const int ig1 = (ieg + 1) % 4, ig2 = ieg + 4;
        double dp[3];
        double leneg = 0.0;
        for (int i = 0; i < 3; ++i) {
            dp[i] = c.v[ig1][i] - c.v[ieg][i];
            leneg += dp[i] * dp[i];
        }
        leneg = std::sqrt(leneg);
        const double dpo[3] = {dp[0] / leneg, dp[1] / leneg, dp[2] / leneg};
        const double leneg_scaled = leneg / (2.0 * nsec1);
        cd zre(0, 0);
        const double delsec = 2.0 / nsec1;
        double secmid = -1.0 - delsec / 2.0;
        for (int is = 0; is < nsec1; ++is) {
            secmid += delsec;
            for (int ig = 0; ig < q.edge_order; ++ig) {
                double sga = secmid + ecx[ig] / nsec1;
                double wga = ecw[ig] * leneg_scaled;
                double d[3];
                for (int i = 0; i < 3; ++i) d[i] = c.v[ieg][i] + dp[i] * (sga + 1.0) / 2.0 - x[i];
                double u[3];
                double dis = normalize3(d, u);
                if (dis < 1e-15) continue;
                cd zg = exp_i(wavruim * dis) / (4.0 * kPi * dis);
                cd zf = zg * cd(-1.0 / dis, wavruim);
                cd zd[3] = {zf * u[0], zf * u[1], zf * u[2]};
                cd w0 = zd[1] * dpo[2] - zd[2] * dpo[1];
                cd w1 = zd[2] * dpo[0] - zd[0] * dpo[2];
                cd w2 = zd[0] * dpo[1] - zd[1] * dpo[0];
                zre += (w0 * nx[0] + w1 * nx[1] + w2 * nx[2]) * wga;
            }
        }
        r.e += zre;
        for (int isec = 0; isec < nsec2; ++isec) {
            const double aresub = 0.25 / nsec2;
            double ss[3] = {0.0, 0.0, 0.0}, ts[3] = {0.0, 0.0, 0.0};
            if (isec == 0) {
                ss[1] = kCsi8[ieg];
                ss[2] = kCsi8[ig2];
                ts[1] = kEta8[ieg];
                ts[2] = kEta8[ig2];
            } else {
                ss[1] = kCsi8[ig2];
                ss[2] = kCsi8[ig1];
                ts[1] = kEta8[ig2];
                ts[2] = kEta8[ig1];
            }
            for (int a = 0; a < q.sub_order; ++a)
                for (int b = 0; b < q.sub_order; ++b) {
                    const double sga = scx[a], tga = scx[b], wei = scw[a] * scw[b];
                    double sgg = 0.5 * (1.0 - sga) * ss[0] + 0.25 * (1.0 + sga) * ((1.0 - tga) * ss[1] + (1.0 + tga) * ss[2]);
                    double tgg = 0.5 * (1.0 - sga) * ts[0] + 0.25 * (1.0 + sga) * ((1.0 - tga) * ts[1] + (1.0 + tga) * ts[2]);
                    double pos[3], jac, ny[3];
                    quad_parameters(c, sgg, tgg, pos, jac, ny);
                    double wga = wei * (1.0 + sga) * aresub * jac;
                    double d[3] = {pos[0] - x[0], pos[1] - x[1], pos[2] - x[2]};
                    double u[3];
                    double dis = normalize3(d, u);
                    if (dis < 1e-15) continue;
                    cd zg = exp_i(wavruim * dis) * (wga / (4.0 * kPi * dis));
                    cd zb = zg * cd(-1.0 / dis, wavruim);
                    double rny = u[0] * ny[0] + u[1] * ny[1] + u[2] * ny[2];
                    double rnx = -(u[0] * nx[0] + u[1] * nx[1] + u[2] * nx[2]);
                    r.g += zg;
                    r.h += zb * rny;
                    r.ht += zb * rnx;
                    double nd = nx[0] * ny[0] + nx[1] * ny[1] + nx[2] * ny[2];
                    r.e += zg * k2 * nd;
                }
        }
    }
    return r;
}

}  // namespace

extern "C" {

// compute_element_geometry (generators.rs:771-850) for Quad4 elements: centre = node average,
// normal from the diagonal cross product (p2 - p0) x (p3 - p1), area = compute_element_area
// (element.rs:326-362, the mean of both diagonal splits).
void or_quad_geometry(int64_t m, const double* nodes, const uint32_t* quads, double* centers, double* normals,
                      double* areas) {
    for (int64_t e = 0; e < m; ++e) {
        const uint32_t* q = quads + 4 * e;
        double p[4][3];
        for (int a = 0; a < 4; ++a)
            for (int j = 0; j < 3; ++j) p[a][j] = nodes[3 * q[a] + j];
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int a = 0; a < 4; ++a) s += p[a][j];
            centers[3 * e + j] = s / 4.0;
        }
        double d1[3], d2[3];
        for (int j = 0; j < 3; ++j) {
            d1[j] = p[2][j] - p[0][j];
            d2[j] = p[3][j] - p[1][j];
        }
        double cr[3] = {d1[1] * d2[2] - d1[2] * d2[1], d1[2] * d2[0] - d1[0] * d2[2], d1[0] * d2[1] - d1[1] * d2[0]};
        double len = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        for (int j = 0; j < 3; ++j) normals[3 * e + j] = len > 1e-15 ? cr[j] / len : 0.0;
        auto sub = [&](int a, int b, double o[3]) {
            for (int j = 0; j < 3; ++j) o[j] = p[a][j] - p[b][j];
        };
        auto clen = [](const double a[3], const double b[3]) {
            double c0 = a[1] * b[2] - a[2] * b[1], c1 = a[2] * b[0] - a[0] * b[2], c2 = a[0] * b[1] - a[1] * b[0];
            return std::sqrt(c0 * c0 + c1 * c1 + c2 * c2);
        };
        double v1[3], v2[3], v3[3], v4[3], v5[3], v6[3];
        sub(1, 0, v1);
        sub(2, 0, v2);
        sub(3, 0, v3);
        sub(2, 1, v4);
        sub(3, 1, v5);
        sub(0, 1, v6);
        const double a1 = 0.5 * clen(v1, v2), a2 = 0.5 * clen(v2, v3), a3 = 0.5 * clen(v4, v5),
                     a4 = 0.5 * clen(v5, v6);
        areas[e] = 0.5 * (a1 + a2 + a3 + a4);
    }
}

// The constant-panel system of a Quad4 mesh (build_tbem_system_with_beta_parallel, tbem.rs:
// 1284-1466, Quad4 branches): A is m x m row-major.
int or_assemble_quad(int64_t n_nodes, const double* nodes, int64_t m, const uint32_t* quads, const or_bc* bc,
                     const or_physics* ph, or_c128 beta_in, int threads, or_c128* A, or_c128* rhs) {
    if (m <= 0) return 1;
    for (int64_t i = 0; i < 4 * m; ++i)
        if (quads[i] >= static_cast<uint64_t>(n_nodes)) return 1;
    std::vector<double> centers(3 * m), normals(3 * m), areas(m);
    or_quad_geometry(m, nodes, quads, centers.data(), normals.data(), areas.data());
    std::vector<Coords4> coords(m);
    for (int64_t e = 0; e < m; ++e)
        for (int a = 0; a < 4; ++a)
            for (int j = 0; j < 3; ++j) coords[e].v[a][j] = nodes[3 * quads[4 * e + a] + j];
    const cd gamma(1.0, 0.0), tau(ph->tau, 0.0), iwr(0.0, ph->pressure_factor);
    const cd beta = C(beta_in);
    std::vector<BcView> bcs(m);
    for (int64_t e = 0; e < m; ++e) bcs[e] = bc_at(bc, e);
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < m; ++i) {
        std::vector<cd> local(m, cd(0, 0));
        cd lrhs(0, 0);
        const BcView& sb = bcs[i];
        if (sb.kind == 0) {
            local[i] -= gamma * 0.5;
            if (sb.has_adm) local[i] -= sb.adm * iwr * beta * tau * 0.5;
            lrhs += sb.value * iwr * beta * tau * 0.5;
        } else if (sb.kind == 1) {
            local[i] += beta * tau * 0.5;
            lrhs -= sb.value * gamma * 0.5;
        }
        const double* x = &centers[3 * i];
        const double* nx = &normals[3 * i];
        for (int64_t j = 0; j < m; ++j) {
            const BcView& fb = bcs[j];
            Channels r = (j == i) ? singular_pair_quad(x, nx, coords[j], *ph)
                                  : regular_pair_quad(x, nx, coords[j], areas[j], *ph);
            cd coeff(0, 0);
            if (fb.kind == 0) {
                coeff = r.h * gamma * tau + r.e * beta;
                if (fb.has_adm) coeff -= (r.g * gamma * tau + r.ht * beta) * fb.adm * iwr;
            } else if (fb.kind == 1) {
                coeff = -(r.g * gamma * tau + r.ht * beta);
            }
            local[j] += coeff;
            if (std::abs(fb.value) > 1e-15) {
                if (fb.kind == 0)
                    lrhs += (r.g * gamma * tau + r.ht * beta) * fb.value * iwr;
                else if (fb.kind == 1)
                    lrhs += (r.h * gamma * tau + r.e * beta) * fb.value;
            }
        }
        for (int64_t j = 0; j < m; ++j) A[i * m + j] = O(local[j]);
        if (rhs) rhs[i] = O(lrhs);
    }
    return 0;
}

}  // extern "C"
