// Quadrature rules and the native (reference-element orthonormal) basis.
#include <cmath>
#include <cstring>

#include "rkdg_internal.hpp"

namespace rkdg {

// Volume rules: barycentric (l0, l1, l2) with weights normalised to 1.
// The 7-point degree-5 rule uses the reference's decimal constants
// (src/triangleinfo.cpp:159-163, 199-205, 219-225) so that the
// reference-native configuration integrates exactly like the reference.
void volume_rule(int nq, double l[][3], double* w) {
    if (nq == 7) {
        const double w1 = 0.797426985353087, w2 = 0.101286507323456;
        const double w3 = 0.059715871789770, w4 = 0.470142064105115;
        const double L[7][3] = {{1.0 / 3, 1.0 / 3, 1.0 / 3}, {w1, w2, w2}, {w2, w1, w2},
                                {w2, w2, w1}, {w3, w4, w4}, {w4, w3, w4}, {w4, w4, w3}};
        const double W[7] = {0.225, 0.125939180544827, 0.125939180544827, 0.125939180544827,
                             0.132394152788506, 0.132394152788506, 0.132394152788506};
        std::memcpy(l, L, sizeof(L));
        std::memcpy(w, W, sizeof(W));
    } else if (nq == 6) {
        // Dunavant's degree-4 six-point rule
        const double a = 0.44594849091596488631832925388305, wa = 0.22338158967801146569500700843312;
        const double b = 0.09157621350977074345957146340220, wb = 0.10995174365532186763832632490021;
        const double L[6][3] = {{1 - 2 * a, a, a}, {a, 1 - 2 * a, a}, {a, a, 1 - 2 * a},
                                {1 - 2 * b, b, b}, {b, 1 - 2 * b, b}, {b, b, 1 - 2 * b}};
        const double W[6] = {wa, wa, wa, wb, wb, wb};
        std::memcpy(l, L, sizeof(L));
        std::memcpy(w, W, sizeof(W));
    } else {
        // Strang-Fix degree-2 three-point rule (interior points)
        const double L[3][3] = {{2.0 / 3, 1.0 / 6, 1.0 / 6}, {1.0 / 6, 2.0 / 3, 1.0 / 6},
                                {1.0 / 6, 1.0 / 6, 2.0 / 3}};
        const double W[3] = {1.0 / 3, 1.0 / 3, 1.0 / 3};
        std::memcpy(l, L, sizeof(L));
        std::memcpy(w, W, sizeof(W));
    }
}

// Gauss-Legendre points as fractions along an edge from its start vertex,
// weights normalised to 1.  The 3-point rule keeps the reference's
// constants (src/triangleinfo.cpp:165, 209-217, 227-232).
void edge_rule(int ng, double* s, double* w) {
    if (ng == 3) {
        const double cp = 0.5 + std::sqrt(15.0) / 10.0;
        s[0] = 1 - cp;
        s[1] = 0.5;
        s[2] = cp;
        w[0] = 0.55555555555556 * 0.5;
        w[1] = 0.88888888888889 * 0.5;
        w[2] = 0.55555555555556 * 0.5;
    } else {
        s[0] = 0.5 - std::sqrt(3.0) / 6.0;
        s[1] = 0.5 + std::sqrt(3.0) / 6.0;
        w[0] = 0.5;
        w[1] = 0.5;
    }
}

namespace {

double factorial(int n) {
    double f = 1;
    for (int i = 2; i <= n; ++i) f *= i;
    return f;
}

// area average of xi^a eta^b over the reference triangle: 2 a! b! / (a+b+2)!
double ref_moment(int a, int b) { return 2.0 * factorial(a) * factorial(b) / factorial(a + b + 2); }

struct NativeBasis {
    double K[6][6];  // psi_i = sum_j K[i][j] m_j, m = 1, xi, eta, xi^2, xi*eta, eta^2
    NativeBasis() {
        const int ex[6][2] = {{0, 0}, {1, 0}, {0, 1}, {2, 0}, {1, 1}, {0, 2}};
        double G[6][6];
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j)
                G[i][j] = ref_moment(ex[i][0] + ex[j][0], ex[i][1] + ex[j][1]);
        // Cholesky G = L L^T; the orthonormal, hierarchical basis is L^-1 m.
        double L[6][6] = {{0}};
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j <= i; ++j) {
                double s = G[i][j];
                for (int k = 0; k < j; ++k) s -= L[i][k] * L[j][k];
                L[i][j] = (i == j) ? std::sqrt(s) : s / L[j][j];
            }
        std::memset(K, 0, sizeof(K));
        for (int i = 0; i < 6; ++i) {  // K = L^-1 by forward substitution
            for (int j = 0; j <= i; ++j) {
                double s = (i == j) ? 1.0 : 0.0;
                for (int k = j; k < i; ++k) s -= L[i][k] * K[k][j];
                K[i][j] = s / L[i][i];
            }
        }
    }
};

const NativeBasis& native() {
    static const NativeBasis nb;
    return nb;
}

}  // namespace

const double (*native_coeff())[6] { return native().K; }

void native_eval(int nbasis, double xi, double eta, double* val, double* dxi, double* deta) {
    const double(*K)[6] = native().K;
    const double m[6] = {1, xi, eta, xi * xi, xi * eta, eta * eta};
    const double mx[6] = {0, 1, 0, 2 * xi, eta, 0};
    const double my[6] = {0, 0, 1, 0, xi, 2 * eta};
    for (int i = 0; i < nbasis; ++i) {
        double v = 0, dx = 0, dy = 0;
        for (int j = 0; j < 6; ++j) {
            v += K[i][j] * m[j];
            dx += K[i][j] * mx[j];
            dy += K[i][j] * my[j];
        }
        if (val) val[i] = v;
        if (dxi) dxi[i] = dx;
        if (deta) deta[i] = dy;
    }
}

RuleTables make_tables(int nq, int ng) {
    RuleTables t;
    std::memset(&t, 0, sizeof(t));
    double l[kMaxNQ][3], w[kMaxNQ];
    volume_rule(nq, l, w);
    for (int q = 0; q < nq; ++q) {
        double v[6], dx[6], dy[6];
        native_eval(6, l[q][1], l[q][2], v, dx, dy);
        for (int i = 0; i < 6; ++i) {
            t.vphi[q][i] = v[i];
            t.vdxi_w[q][i] = w[q] * dx[i];
            t.veta_w[q][i] = w[q] * dy[i];
        }
        t.vw[q] = w[q];
    }
    double s[kMaxNG], ew[kMaxNG];
    edge_rule(ng, s, ew);
    // reference-element edges: 0 = (1,0)->(0,1), 1 = (0,1)->(0,0), 2 = (0,0)->(1,0)
    for (int k = 0; k < 3; ++k)
        for (int g = 0; g < ng; ++g) {
            double xi, eta;
            if (k == 0) {
                xi = 1 - s[g];
                eta = s[g];
            } else if (k == 1) {
                xi = 0;
                eta = 1 - s[g];
            } else {
                xi = s[g];
                eta = 0;
            }
            double v[6];
            native_eval(6, xi, eta, v, nullptr, nullptr);
            for (int i = 0; i < 6; ++i) t.ephi[k][g][i] = v[i];
        }
    for (int g = 0; g < ng; ++g) t.ew[g] = ew[g];
    // P1 part at the edge midpoints, and its least-squares inverse
    const double mid[3][2] = {{0.5, 0.5}, {0.0, 0.5}, {0.5, 0.0}};
    for (int k = 0; k < 3; ++k) {
        double v[6];
        native_eval(3, mid[k][0], mid[k][1], v, nullptr, nullptr);
        t.mphi[k][0] = v[1];
        t.mphi[k][1] = v[2];
    }
    double a11 = 0, a12 = 0, a22 = 0;
    for (int k = 0; k < 3; ++k) {
        a11 += t.mphi[k][0] * t.mphi[k][0];
        a12 += t.mphi[k][0] * t.mphi[k][1];
        a22 += t.mphi[k][1] * t.mphi[k][1];
    }
    double det = a11 * a22 - a12 * a12;
    for (int k = 0; k < 3; ++k) {
        t.minv[0][k] = (a22 * t.mphi[k][0] - a12 * t.mphi[k][1]) / det;
        t.minv[1][k] = (a11 * t.mphi[k][1] - a12 * t.mphi[k][0]) / det;
    }
    return t;
}

}  // namespace rkdg

extern "C" int rkdg_native_basis(int32_t nbasis, int32_t npts, const double* xi, const double* eta,
                                 double* out) {
    if (nbasis < 1 || nbasis > 6 || npts < 0 || (npts > 0 && (!xi || !eta || !out))) {
        rkdg::set_error("rkdg_native_basis: invalid arguments");
        return RKDG_ERR_INVALID;
    }
    for (int p = 0; p < npts; ++p) rkdg::native_eval(nbasis, xi[p], eta[p], out + (size_t)p * nbasis,
                                                     nullptr, nullptr);
    return RKDG_OK;
}
