// Host-side mesh ingest, connectivity, locality ordering and FP64 geometry.
//
// Replaces the reference's CUnstructuredGrid set-up (src/unstructuredgrid.cpp)
// and CTriangleInfo (src/triangleinfo.cpp) for one device: connectivity is
// built by sorting edge keys (O(T log T)) instead of the reference's O(T^2)
// searches (src/unstructuredgrid.cpp:88-107, 164-191, 307-318), boundary
// conditions are per-edge tags instead of ghost cells, and the partition
// file's role reduces to a locality-preserving (Morton) element order.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <numeric>
#include <sstream>

#include "rkdg_internal.hpp"

namespace rkdg {

uint32_t pack_info(const int8_t* shared3, const int8_t* bc3, uint32_t lim_pair) {
    uint32_t w = 0;
    for (int k = 0; k < 3; ++k) {
        uint32_t s = shared3[k] < 0 ? 3u : (uint32_t)shared3[k];
        w |= (s & 3u) << (2 * k);
        w |= ((uint32_t)bc3[k] & 3u) << (6 + 2 * k);
    }
    return w | ((lim_pair & 7u) << 12);
}

void upload_limiter(void* dev, int ld, int64_t e0, const std::vector<double>& lim, int T, int prec,
                    cudaStream_t stream) {
    const size_t w = prec == RKDG_FP64 ? 16 : 8;  // double2 or float2 per element and edge
    std::vector<unsigned char> rows((size_t)3 * T * w);
    for (int k = 0; k < 3; ++k)
        for (int t = 0; t < T; ++t) {
            unsigned char* d = rows.data() + ((size_t)k * T + t) * w;
            const double a = lim[(size_t)6 * t + 2 * k], b = lim[(size_t)6 * t + 2 * k + 1];
            if (prec == RKDG_FP64) {
                std::memcpy(d, &a, 8);
                std::memcpy(d + 8, &b, 8);
            } else {
                const float af = (float)a, bf = (float)b;
                std::memcpy(d, &af, 4);
                std::memcpy(d + 4, &bf, 4);
            }
        }
    RKDG_CUDA_TRY(cudaMemcpy2DAsync(static_cast<unsigned char*>(dev) + (size_t)e0 * w, (size_t)ld * w, rows.data(),
                                    (size_t)T * w, (size_t)T * w, 3, cudaMemcpyHostToDevice, stream));
    RKDG_CUDA_TRY(cudaStreamSynchronize(stream));  // the host rows are temporaries
}

HostMesh build_mesh(const rkdg_mesh_desc& d) {
    if (d.ntri <= 0 || d.nvert <= 0 || !d.vertices || !d.tri_vertex)
        throw Error{RKDG_ERR_INVALID, "mesh: ntri, nvert, vertices and tri_vertex are required"};
    const int T = d.ntri;
    HostMesh m;
    m.T = T;
    m.xy.resize((size_t)6 * T);
    m.tri_vertex.assign(d.tri_vertex, d.tri_vertex + (size_t)3 * T);
    m.vertices.assign(d.vertices, d.vertices + (size_t)2 * d.nvert);
    for (int t = 0; t < T; ++t) {
        for (int k = 0; k < 3; ++k) {
            int v = d.tri_vertex[3 * t + k];
            if (v < 0 || v >= d.nvert)
                throw Error{RKDG_ERR_INVALID, "mesh: vertex id out of range in triangle " +
                                                  std::to_string(t)};
            m.xy[6 * t + 2 * k] = d.vertices[2 * v];
            m.xy[6 * t + 2 * k + 1] = d.vertices[2 * v + 1];
        }
        const double* p = &m.xy[6 * t];
        double det = (p[2] - p[0]) * (p[5] - p[1]) - (p[3] - p[1]) * (p[4] - p[0]);
        if (!(det > 0))
            throw Error{RKDG_ERR_INVALID, "mesh: triangle " + std::to_string(t) +
                                              " is not counter-clockwise or is degenerate"};
    }
    // neighbours
    m.nbr.assign((size_t)3 * T, -1);
    if (d.tri_neighbour) {
        for (size_t i = 0; i < (size_t)3 * T; ++i) {
            int n = d.tri_neighbour[i];
            if (n < -1 || n >= T) throw Error{RKDG_ERR_INVALID, "mesh: neighbour id out of range"};
            m.nbr[i] = n;
        }
    } else {
        // sort the 3T edge keys (min vertex, max vertex); equal neighbours pair up
        std::vector<std::pair<uint64_t, int32_t>> keys((size_t)3 * T);
        for (int t = 0; t < T; ++t)
            for (int k = 0; k < 3; ++k) {
                uint64_t a = (uint32_t)d.tri_vertex[3 * t + (k + 1) % 3];
                uint64_t b = (uint32_t)d.tri_vertex[3 * t + (k + 2) % 3];
                if (a > b) std::swap(a, b);
                keys[(size_t)3 * t + k] = {(a << 32) | b, 3 * t + k};
            }
        std::sort(keys.begin(), keys.end());
        for (size_t i = 0; i + 1 < keys.size();) {
            if (keys[i].first == keys[i + 1].first) {
                if (i + 2 < keys.size() && keys[i + 2].first == keys[i].first)
                    throw Error{RKDG_ERR_INVALID, "mesh: edge shared by more than two triangles"};
                int e0 = keys[i].second, e1 = keys[i + 1].second;
                m.nbr[e0] = e1 / 3;
                m.nbr[e1] = e0 / 3;
                i += 2;
            } else {
                ++i;
            }
        }
    }
    // neighbour-local index of each shared edge (src/unstructuredgrid.cpp:934-976)
    m.shared.assign((size_t)3 * T, -1);
    for (int t = 0; t < T; ++t)
        for (int k = 0; k < 3; ++k) {
            int n = m.nbr[3 * t + k];
            if (n < 0) continue;
            int found = -1;
            for (int j = 0; j < 3; ++j)
                if (m.nbr[3 * n + j] == t) {
                    if (found >= 0 && n != t)
                        throw Error{RKDG_ERR_INVALID, "mesh: triangles " + std::to_string(t) +
                                                          " and " + std::to_string(n) +
                                                          " share more than one edge"};
                    found = j;
                }
            if (found < 0)
                throw Error{RKDG_ERR_INVALID, "mesh: neighbour relation is not symmetric at triangle " +
                                                  std::to_string(t)};
            m.shared[3 * t + k] = (int8_t)found;
        }
    // boundary tags
    m.bc.assign((size_t)3 * T, 0);
    for (int t = 0; t < T; ++t)
        for (int k = 0; k < 3; ++k) {
            if (m.nbr[3 * t + k] >= 0) continue;
            int tag;
            if (d.bc) {
                tag = d.bc[3 * t + k];
                if (tag < 1 || tag > 3)
                    throw Error{RKDG_ERR_INVALID, "mesh: boundary edge without a valid tag at triangle " +
                                                      std::to_string(t)};
            } else {
                // the reference's rule: ghost triangle = the reflection of this
                // one's opposite vertex through the edge midpoint
                // (src/unstructuredgrid.cpp:527-559); far field when its
                // barycentre lies outside |x|,|y| <= 15, else wall (:729-760)
                const double* p = &m.xy[6 * t];
                int a = (k + 1) % 3, b = (k + 2) % 3;
                double gx = p[2 * a] + p[2 * b] - p[2 * k];
                double gy = p[2 * a + 1] + p[2 * b + 1] - p[2 * k + 1];
                double bx = (gx + p[2 * a] + p[2 * b]) / 3.0;
                double by = (gy + p[2 * a + 1] + p[2 * b + 1]) / 3.0;
                bool far = bx < -15.0 || bx > 15.0 || by < -15.0 || by > 15.0;
                tag = far ? RKDG_BC_FARFIELD : RKDG_BC_REFLECTION;
            }
            m.bc[3 * t + k] = (int8_t)tag;
        }
    m.perm.resize(T);
    std::iota(m.perm.begin(), m.perm.end(), 0);
    return m;
}

std::vector<int32_t> morton_order(const HostMesh& m) {
    const int T = m.T;
    std::vector<double> cx(T), cy(T);
    double x0 = 1e300, y0 = 1e300, x1 = -1e300, y1 = -1e300;
    for (int t = 0; t < T; ++t) {
        const double* p = &m.xy[6 * t];
        cx[t] = (p[0] + p[2] + p[4]) / 3;
        cy[t] = (p[1] + p[3] + p[5]) / 3;
        x0 = std::min(x0, cx[t]);
        x1 = std::max(x1, cx[t]);
        y0 = std::min(y0, cy[t]);
        y1 = std::max(y1, cy[t]);
    }
    double sx = x1 > x0 ? 65535.0 / (x1 - x0) : 0, sy = y1 > y0 ? 65535.0 / (y1 - y0) : 0;
    auto spread = [](uint32_t v) {
        uint64_t x = v & 0xFFFFu;
        x = (x | (x << 8)) & 0x00FF00FFu;
        x = (x | (x << 4)) & 0x0F0F0F0Fu;
        x = (x | (x << 2)) & 0x33333333u;
        x = (x | (x << 1)) & 0x55555555u;
        return x;
    };
    std::vector<std::pair<uint64_t, int32_t>> key(T);
    for (int t = 0; t < T; ++t) {
        uint32_t qx = (uint32_t)std::min(65535.0, (cx[t] - x0) * sx);
        uint32_t qy = (uint32_t)std::min(65535.0, (cy[t] - y0) * sy);
        key[t] = {spread(qx) | (spread(qy) << 1), t};
    }
    std::sort(key.begin(), key.end());
    std::vector<int32_t> perm(T);
    for (int t = 0; t < T; ++t) perm[t] = key[t].second;
    return perm;
}

HostMesh permute_mesh(const HostMesh& m, const std::vector<int32_t>& perm) {
    const int T = m.T;
    std::vector<int32_t> inv(T);
    for (int i = 0; i < T; ++i) inv[perm[i]] = i;
    HostMesh r;
    r.T = T;
    r.xy.resize(m.xy.size());
    r.nbr.resize(m.nbr.size());
    r.bc.resize(m.bc.size());
    r.shared.resize(m.shared.size());
    r.perm.resize(T);
    for (int i = 0; i < T; ++i) {
        int o = perm[i];
        std::memcpy(&r.xy[6 * i], &m.xy[6 * o], 6 * sizeof(double));
        for (int k = 0; k < 3; ++k) {
            int n = m.nbr[3 * o + k];
            r.nbr[3 * i + k] = n >= 0 ? inv[n] : -1;
            r.bc[3 * i + k] = m.bc[3 * o + k];
            r.shared[3 * i + k] = m.shared[3 * o + k];
        }
        r.perm[i] = m.perm[o];
    }
    r.tri_vertex = m.tri_vertex;
    r.vertices = m.vertices;
    return r;
}

namespace {

// Symmetric positive definite solve (Cholesky) of the n x n system G c = r.
void spd_solve(int n, const double* G, int ldg, double* r) {
    double L[6][6] = {{0}};
    for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = G[i * ldg + j];
            for (int k = 0; k < j; ++k) s -= L[i][k] * L[j][k];
            L[i][j] = (i == j) ? std::sqrt(s) : s / L[j][j];
        }
    for (int i = 0; i < n; ++i) {
        double s = r[i];
        for (int k = 0; k < i; ++k) s -= L[i][k] * r[k];
        r[i] = s / L[i][i];
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = r[i];
        for (int k = i + 1; k < n; ++k) s -= L[k][i] * r[k];
        r[i] = s / L[i][i];
    }
}

// The reference's per-element basis (src/triangleinfo.cpp:281-602): basis k
// is the monomial k of (X, Y) = ((x - xc), (y - yc)) / sqrt(area) in the
// order 1, X, Y, X^2, XY, Y^2, minus its area-average projection on the
// earlier monomials.  Returns coefficients on the scaled monomials.
void reference_basis_scaled(const double* p, double area, double xc, double yc, double c[6][6]) {
    double l[kMaxNQ][3], w[kMaxNQ];
    volume_rule(6, l, w);  // degree 4: exact for products of quadratics
    const double s = 1.0 / std::sqrt(area);
    double G[6][6] = {{0}};
    for (int q = 0; q < 6; ++q) {
        double x = l[q][0] * p[0] + l[q][1] * p[2] + l[q][2] * p[4];
        double y = l[q][0] * p[1] + l[q][1] * p[3] + l[q][2] * p[5];
        double X = (x - xc) * s, Y = (y - yc) * s;
        double m[6] = {1, X, Y, X * X, X * Y, Y * Y};
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) G[i][j] += w[q] * m[i] * m[j];
    }
    std::memset(c, 0, sizeof(double) * 36);
    c[0][0] = 1;
    for (int k = 1; k < 6; ++k) {
        double r[6];
        for (int i = 0; i < k; ++i) r[i] = -G[i][k];
        spd_solve(k, &G[0][0], 6, r);
        for (int j = 0; j < k; ++j) c[k][j] = r[j];
        c[k][k] = 1;
    }
}

}  // namespace

HostGeometry build_geometry(const HostMesh& m, int order, bool with_conversion, bool with_limiter) {
    const int T = m.T;
    HostGeometry g;
    g.jinv.resize((size_t)4 * T);
    g.area.resize(T);
    if (with_conversion) {
        g.conv_in.assign((size_t)36 * T, 0.0);
        g.conv_out.assign((size_t)36 * T, 0.0);
    }
    if (with_limiter) {
        g.lim.assign((size_t)6 * T, 0.0);
        g.lim_pair.assign(T, 0);
    }
    double l[kMaxNQ][3], w[kMaxNQ];
    volume_rule(6, l, w);
    double psi[6][6];  // native basis at the 6 rule points
    for (int q = 0; q < 6; ++q) native_eval(6, l[q][1], l[q][2], psi[q], nullptr, nullptr);
    (void)order;

    for (int t = 0; t < T; ++t) {
        const double* p = &m.xy[6 * t];
        double ax = p[2] - p[0], ay = p[3] - p[1], bx = p[4] - p[0], by = p[5] - p[1];
        double det = ax * by - ay * bx;
        g.jinv[4 * t + 0] = by / det;
        g.jinv[4 * t + 1] = -bx / det;
        g.jinv[4 * t + 2] = -ay / det;
        g.jinv[4 * t + 3] = ax / det;
        // area as the reference computes it (src/triangleinfo.cpp:171)
        double area = 0.5 * std::fabs((p[4] - p[0]) * (p[3] - p[1]) - (p[5] - p[1]) * (p[2] - p[0]));
        g.area[t] = area;
        if (with_conversion) {
            double xc = (p[0] + p[2] + p[4]) / 3.0, yc = (p[1] + p[3] + p[5]) / 3.0;
            double c[6][6];
            reference_basis_scaled(p, area, xc, yc, c);
            const double s = 1.0 / std::sqrt(area);
            // C[i][j] = area average of phi_i psi_j (phi_i = sum_j C[i][j] psi_j)
            double C[6][6] = {{0}};
            for (int q = 0; q < 6; ++q) {
                double x = l[q][0] * p[0] + l[q][1] * p[2] + l[q][2] * p[4];
                double y = l[q][0] * p[1] + l[q][1] * p[3] + l[q][2] * p[5];
                double X = (x - xc) * s, Y = (y - yc) * s;
                double mm[6] = {1, X, Y, X * X, X * Y, Y * Y};
                for (int i = 0; i < 6; ++i) {
                    double phi = 0;
                    for (int j = 0; j <= i; ++j) phi += c[i][j] * mm[j];
                    for (int j = 0; j < 6; ++j) C[i][j] += w[q] * phi * psi[q][j];
                }
            }
            const int nb = order == 1 ? 3 : 6;
            for (int i = 0; i < 6; ++i) {
                double sq = 0;  // area average of phi_i^2
                for (int j = 0; j < nb; ++j) sq += C[i][j] * C[i][j];
                for (int j = 0; j < 6; ++j) {
                    g.conv_in[(size_t)36 * t + 6 * i + j] = (i < nb && j < nb) ? C[i][j] : 0.0;
                    g.conv_out[(size_t)36 * t + 6 * i + j] =
                        (i < nb && j < nb) ? C[i][j] / sq : 0.0;
                }
            }
        }
    }
    if (with_limiter) {
        // Cockburn & Shu (1998, J. Comput. Phys. 141:199-224, sec. 2.4) geometry
        // per edge k: (alpha, beta) and the pairing edge j with
        // m_k - b0 = alpha (b_k - b0) + beta (b_j - b0); the direction
        // m_k - b0 and its length (the TVB threshold scale) are formed on the
        // device from J^-1.
        for (int t = 0; t < T; ++t) {
            const double* p = &m.xy[6 * t];
            double b0x = (p[0] + p[2] + p[4]) / 3.0, b0y = (p[1] + p[3] + p[5]) / 3.0;
            double bx[3], by[3], mx[3], my[3];
            for (int k = 0; k < 3; ++k) {
                int a = (k + 1) % 3, b = (k + 2) % 3;
                mx[k] = 0.5 * (p[2 * a] + p[2 * b]);
                my[k] = 0.5 * (p[2 * a + 1] + p[2 * b + 1]);
                int n = m.nbr[3 * t + k];
                if (n >= 0) {
                    int se = m.shared[3 * t + k];
                    const double* q = &m.xy[6 * n];
                    int na = (se + 1) % 3, nbv = (se + 2) % 3;
                    double nmx = 0.5 * (q[2 * na] + q[2 * nbv]), nmy = 0.5 * (q[2 * na + 1] + q[2 * nbv + 1]);
                    double nbx = (q[0] + q[2] + q[4]) / 3.0, nby = (q[1] + q[3] + q[5]) / 3.0;
                    bx[k] = mx[k] + (nbx - nmx);
                    by[k] = my[k] + (nby - nmy);
                } else {
                    double ex = p[2 * b] - p[2 * a], ey = p[2 * b + 1] - p[2 * a + 1];
                    double len = std::sqrt(ex * ex + ey * ey);
                    double nx = ey / len, ny = -ex / len;
                    double dd = (mx[k] - b0x) * nx + (my[k] - b0y) * ny;
                    bx[k] = b0x + 2 * dd * nx;
                    by[k] = b0y + 2 * dd * ny;
                }
            }
            for (int k = 0; k < 3; ++k) {
                double rx = mx[k] - b0x, ry = my[k] - b0y;
                double best = -1e300, ba = 0, bb = 0;
                int bj = (k + 1) % 3;
                for (int s = 1; s <= 2; ++s) {
                    int j = (k + s) % 3;
                    double ax = bx[k] - b0x, ay = by[k] - b0y, cx = bx[j] - b0x, cy = by[j] - b0y;
                    double det = ax * cy - ay * cx;
                    if (std::fabs(det) < 1e-300) continue;
                    double al = (rx * cy - ry * cx) / det, be = (ax * ry - ay * rx) / det;
                    double sc = std::min(al, be);
                    if (sc > best + 1e-14) {
                        best = sc;
                        ba = al;
                        bb = be;
                        bj = j;
                    }
                }
                g.lim[(size_t)6 * t + 2 * k] = ba;
                g.lim[(size_t)6 * t + 2 * k + 1] = bb;
                if (bj == (k + 2) % 3) g.lim_pair[t] |= (uint8_t)(1u << k);
            }
        }
    }
    return g;
}

TileTables build_tiles(const HostMesh& m, int elem_offset, int sid, int order, int halo_offset,
                       int task_offset, int n_tiled, int tile) {
    const int T = n_tiled >= 0 ? n_tiled : m.T, B = tile;
    if (B != 128 && B != 256) throw Error{RKDG_ERR_INVALID, "tiles hold 128 or 256 elements"};
    TileTables t;
    t.tile = B;
    t.ntiles = (T + B - 1) / B;
    t.code.assign((size_t)4 * m.T, 0);
    t.desc.assign((size_t)8 * t.ntiles, 0);
    int maxh = 0;
    for (int tile = 0; tile < t.ntiles; ++tile) {
        const int e0 = tile * B, e1 = std::min(T, e0 + B);
        const int h_begin = (int)(t.halo.size() / 2), k_begin = (int)t.task.size();
        int nh = 0;
        for (int k = 0; k < 3; ++k)  // tasks and halo slots sorted by edge, then element
            for (int e = e0; e < e1; ++e) {
                const int le = e - e0;
                const int n = m.nbr[3 * e + k];
                int code;
                bool task = true;
                if (n < 0) {
                    code = EDGE_BOUNDARY | ((m.bc[3 * e + k] & 3) << 2);
                } else if (n >= e0 && n < e1) {
                    const int se = m.shared[3 * e + k];
                    const bool owner = e < n;
                    code = (owner ? EDGE_IN_OWNER : EDGE_IN_OTHER) | (se << 2) | ((n - e0) << 4);
                    task = owner;
                } else {
                    const int se = m.shared[3 * e + k];
                    code = EDGE_HALO | (se << 2) | (nh << 4);
                    t.halo.push_back(elem_offset + n);
                    t.halo.push_back(se);
                    ++nh;
                }
                t.code[(size_t)4 * e + k] = code;
                if (task) t.task.push_back((uint16_t)(le * 4 + k));
            }
        maxh = std::max(maxh, nh);
        int32_t* d = &t.desc[(size_t)8 * tile];
        d[0] = elem_offset + e0;
        d[1] = e1 - e0;
        d[2] = sid;
        d[3] = order;
        d[4] = halo_offset + h_begin;
        d[5] = nh;
        d[6] = task_offset + k_begin;
        d[7] = (int)t.task.size() - k_begin;
    }
    t.max_halo = std::max(4, (maxh + 3) / 4 * 4);
    return t;
}

}  // namespace rkdg

// ------------------------------------------------------------ file input --
namespace {

// key value [# comment] lines, as the reference's CConfig (src/config.cpp:57-112)
std::map<std::string, std::string> parse_conf(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw rkdg::Error{RKDG_ERR_IO, "cannot open " + path};
    std::map<std::string, std::string> kv;
    std::string line;
    while (std::getline(f, line)) {
        size_t a = line.find_first_not_of(" \t\r");
        if (a == std::string::npos || line[a] == '#') continue;
        size_t b = line.find_first_of(" =\t", a);
        if (b == std::string::npos) continue;
        size_t c = line.find_first_not_of(" =\t", b);
        if (c == std::string::npos) continue;
        size_t e = line.find_first_of(",; #\t\r", c);
        kv[line.substr(a, b - a)] = line.substr(c, e == std::string::npos ? std::string::npos : e - c);
    }
    return kv;
}

// Reads whitespace-separated numbers, skipping a first line that does not
// start with a number (the '#...' header lines of the reference's files).
template <class T>
std::vector<T> read_numbers(const std::string& path, size_t want) {
    std::ifstream f(path);
    if (!f) throw rkdg::Error{RKDG_ERR_IO, "cannot open " + path};
    std::string first;
    std::streampos start = f.tellg();
    std::getline(f, first);
    size_t a = first.find_first_not_of(" \t\r");
    bool header = a != std::string::npos && !(std::isdigit((unsigned char)first[a]) ||
                                              first[a] == '-' || first[a] == '+' || first[a] == '.');
    if (!header) {
        f.clear();
        f.seekg(start);
    }
    std::vector<T> v;
    v.reserve(want);
    T x;
    while (v.size() < want && (f >> x)) v.push_back(x);
    if (v.size() < want)
        throw rkdg::Error{RKDG_ERR_IO, path + ": expected " + std::to_string(want) + " numbers, read " +
                                           std::to_string(v.size())};
    return v;
}

}  // namespace

extern "C" int rkdg_read_mesh(const char* base_dir, const char* mesh_conf, rkdg_mesh_desc* out) {
    try {
        if (!base_dir || !mesh_conf || !out) throw rkdg::Error{RKDG_ERR_INVALID, "rkdg_read_mesh: null argument"};
        std::string base(base_dir);
        if (!base.empty() && base.back() != '/') base += '/';
        auto kv = parse_conf(base + mesh_conf);
        auto get = [&](const char* k) {
            auto it = kv.find(k);
            if (it == kv.end()) throw rkdg::Error{RKDG_ERR_IO, std::string("mesh configuration lacks ") + k};
            return it->second;
        };
        int T = std::atoi(get("trianglenum").c_str());
        int V = std::atoi(get("verticenum").c_str());
        if (T <= 0 || V <= 0) throw rkdg::Error{RKDG_ERR_IO, "mesh configuration: bad sizes"};
        auto verts = read_numbers<double>(base + get("vertice_filename"), (size_t)2 * V);
        auto tv = read_numbers<long long>(base + get("trivertice_filename"), (size_t)3 * T);
        long long vmin = *std::min_element(tv.begin(), tv.end());
        long long vmax = *std::max_element(tv.begin(), tv.end());
        bool one_based = vmin >= 1 && vmax == V;
        std::vector<long long> nb;
        bool have_nb = kv.count("trineigh_filename") > 0;
        if (have_nb) {
            try {
                nb = read_numbers<long long>(base + get("trineigh_filename"), (size_t)3 * T);
            } catch (const rkdg::Error&) {
                have_nb = false;  // rebuilt from the vertices below
            }
        }
        out->ntri = T;
        out->nvert = V;
        double* vv = (double*)std::malloc(sizeof(double) * 2 * V);
        int32_t* tt = (int32_t*)std::malloc(sizeof(int32_t) * 3 * T);
        int32_t* nn = have_nb ? (int32_t*)std::malloc(sizeof(int32_t) * 3 * T) : nullptr;
        std::copy(verts.begin(), verts.end(), vv);
        for (size_t i = 0; i < tv.size(); ++i) tt[i] = (int32_t)(tv[i] - (one_based ? 1 : 0));
        if (nn)
            for (size_t i = 0; i < nb.size(); ++i) {
                long long x = nb[i] - (one_based ? 1 : 0);
                nn[i] = (int32_t)(x < 0 ? -1 : x);
            }
        out->vertices = vv;
        out->tri_vertex = tt;
        out->tri_neighbour = nn;
        out->bc = nullptr;
        return RKDG_OK;
    } catch (const rkdg::Error& e) {
        rkdg::set_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        rkdg::set_error(e.what());
        return RKDG_ERR_IO;
    }
}

extern "C" void rkdg_free_mesh(rkdg_mesh_desc* m) {
    if (!m) return;
    std::free((void*)m->vertices);
    std::free((void*)m->tri_vertex);
    std::free((void*)m->tri_neighbour);
    std::free((void*)m->bc);
    std::memset(m, 0, sizeof(*m));
}

extern "C" int rkdg_build_connectivity(const rkdg_mesh_desc* mesh, int32_t* neighbour, int8_t* shared,
                                       int8_t* bc) {
    try {
        if (!mesh) throw rkdg::Error{RKDG_ERR_INVALID, "null mesh"};
        rkdg::HostMesh m = rkdg::build_mesh(*mesh);
        if (neighbour) std::copy(m.nbr.begin(), m.nbr.end(), neighbour);
        if (shared) std::copy(m.shared.begin(), m.shared.end(), shared);
        if (bc) std::copy(m.bc.begin(), m.bc.end(), bc);
        return RKDG_OK;
    } catch (const rkdg::Error& e) {
        rkdg::set_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        rkdg::set_error(e.what());
        return RKDG_ERR_INVALID;
    }
}

extern "C" int rkdg_locality_order(const rkdg_mesh_desc* mesh, int32_t* perm) {
    try {
        if (!mesh || !perm) throw rkdg::Error{RKDG_ERR_INVALID, "null argument"};
        rkdg::HostMesh m = rkdg::build_mesh(*mesh);
        std::vector<int32_t> p = rkdg::morton_order(m);
        std::copy(p.begin(), p.end(), perm);
        return RKDG_OK;
    } catch (const rkdg::Error& e) {
        rkdg::set_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        rkdg::set_error(e.what());
        return RKDG_ERR_INVALID;
    }
}
