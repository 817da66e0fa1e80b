// Host mesh builder: produces the o_MESH arrays of the reference from a node
// list and an element list.  Every routine below restates one reference
// routine; floating-point expressions keep the reference's operand order so
// that the arrays are bit-identical to what the Fortran driver computes
// (compiled without FMA contraction).
//
//   read_mesh_ser        src/fv_main.F90:787-945
//   test_elem            src/fv_mesh_array.F90:1-82
//   find_edges           src/fv_mesh_array.F90:395-718
//   edge_center          src/fv_mesh_array.F90:720-740
//   elem_center          src/fv_mesh_array.F90:742-789
//   find_elem_neighbors  src/fv_mesh_array.F90:791-946
//   mesh_arrays1         src/fv_mesh_array.F90:948-1139
//   cdiff                src/fv_mesh_array.F90:1141-1152
//   mesh_arrays2         src/fv_mesh_array.F90:1155-1386
//   find_up_downwind_triangles src/fv_mesh_array.F90:1390-1618
//   SET_SIGMA            src/fv_vert_coord.F90:135-280 (cases 1, 2)
//   a_tp                 src/fv_ini.F90:94-107
#include "fesomc_gpu.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

namespace {

const double kPi = 3.14159265358979;          // fv_var.F90:8 (as written)
const double kRad = kPi / 180.0;
const double kREarth = 6400000.0;
const double kOmega = 2.0 * kPi / (3600.0 * 24.0);

}  // namespace

struct fesomc_mesh_builder {
    int nod2D = 0, elem2D = 0, edge2D = 0, edge2D_in = 0, elem2D_tri = 0;
    int nsigma = 0, nie_max = 0;
    bool cartesian = false;
    double cyclic_length = 0.0;
    // all connectivity stored 1-based, Fortran layout
    std::vector<int32_t> index_nod2D, elem2D_nodes, edge_nodes, edge_tri,
        elem_edges, elem_neighbors, nod_in_elem2D_num, nod_in_elem2D,
        edge_up_dn_tri, in_obn, nod_rivers;
    std::vector<double> coord, depth, area, elem_area, elem_cos, coriolis,
        metric_factor, w_cv, gradient_sca, gradient_vec, edge_dxdy,
        edge_cross_dxdy, sigma, a_tp, ac, center_x, center_y;
    bool have_up_dn = false;

    // 1-based accessors
    int en(int q, int e) const { return elem2D_nodes[4 * (e - 1) + (q - 1)]; }
    double cx(int n) const { return coord[2 * (n - 1)]; }
    double cy(int n) const { return coord[2 * (n - 1) + 1]; }

    void elem_center(int elem, double &x, double &y, double &s) const;
    void edge_center(int n1, int n2, double &x, double &y) const;
    double cfix(double d) const {
        if (d > cyclic_length / 2.0) d = d - cyclic_length;
        if (d < -cyclic_length / 2.0) d = d + cyclic_length;
        return d;
    }
};

void fesomc_mesh_builder::edge_center(int n1, int n2, double &x, double &y) const {
    double a0 = cx(n1), a1 = cy(n1), b0 = cx(n2), b1 = cy(n2);
    if (a0 - b0 > cyclic_length / 2.0) a0 = a0 - cyclic_length;
    if (a0 - b0 < -cyclic_length / 2.0) b0 = b0 - cyclic_length;
    x = 0.5 * (a0 + b0);
    y = 0.5 * (a1 + b1);
}

void fesomc_mesh_builder::elem_center(int elem, double &x, double &y, double &s) const {
    int nd[4] = {en(1, elem), en(2, elem), en(3, elem), en(4, elem)};
    double ax[4], ay[4];
    for (int k = 0; k < 4; ++k) { ax[k] = cx(nd[k]); ay[k] = cy(nd[k]); }
    if (nd[0] == nd[3]) {
        double amin = ax[0];
        for (int k = 1; k < 3; ++k) if (ax[k] < amin) amin = ax[k];
        for (int k = 0; k < 3; ++k)
            if (ax[k] - amin > cyclic_length / 2.0) ax[k] = ax[k] - cyclic_length;
        x = ((ax[0] + ax[1]) + ax[2]) / 3.0;
        y = ((ay[0] + ay[1]) + ay[2]) / 3.0;
        s = 0.5 * std::fabs((ax[1] - ax[0]) * (ay[2] - ay[0]) - (ay[1] - ay[0]) * (ax[2] - ax[0]));
    } else {
        double amin = ax[0];
        for (int k = 1; k < 4; ++k) if (ax[k] < amin) amin = ax[k];
        for (int k = 0; k < 4; ++k)
            if (ax[k] - amin > cyclic_length / 2.0) ax[k] = ax[k] - cyclic_length;
        double xx = (ax[0] + ax[2]) + ax[3];
        double yy = (ay[0] + ay[2]) + ay[3];
        double x1 = (ax[0] + ax[1]) + ax[2];
        double y1 = (ay[0] + ay[1]) + ay[2];
        double s1 = std::fabs((ax[2] - ax[3]) * (ay[0] - ay[3]) - (ay[2] - ay[3]) * (ax[0] - ax[3]));
        double s2 = std::fabs((ax[2] - ax[1]) * (ay[0] - ay[1]) - (ay[2] - ay[1]) * (ax[0] - ax[1]));
        x = ((xx * s1 + x1 * s2) / 3.0) / (s1 + s2);
        y = ((yy * s1 + y1 * s2) / 3.0) / (s1 + s2);
        s = 0.5 * (s1 + s2);
    }
}

namespace {

// test_elem: make the node order of every element clockwise.
int test_elem(fesomc_mesh_builder &b) {
    for (int n = 1; n <= b.elem2D; ++n) {
        int32_t *el = &b.elem2D_nodes[4 * (n - 1)];
        double a0 = b.cx(el[0]), a1 = b.cy(el[0]);
        if (el[0] == el[3]) {
            double b0 = b.cfix(b.cx(el[1]) - a0), b1 = b.cy(el[1]) - a1;
            double c0 = b.cfix(b.cx(el[2]) - a0), c1 = b.cy(el[2]) - a1;
            double r = b0 * c1 - b1 * c0;
            if (r > 0.0) std::swap(el[1], el[2]);
        } else {
            double b0 = b.cfix(b.cx(el[1]) - a0), b1 = b.cy(el[1]) - a1;
            double c0 = b.cfix(b.cx(el[2]) - a0), c1 = b.cy(el[2]) - a1;
            double d0 = b.cfix(b.cx(el[3]) - a0), d1 = b.cy(el[3]) - a1;
            double r = b0 * c1 - b1 * c0;
            double r1 = b0 * d1 - b1 * d0;
            if (r1 * r < 0.0) return FESOMC_EMESH;
            if (r > 0) std::swap(el[1], el[3]);
        }
    }
    return FESOMC_OK;
}

// find_edges (a)-(e)
void find_edges(fesomc_mesh_builder &b) {
    const int N = b.nod2D, E = b.elem2D;
    std::vector<int> ne_num(N + 1, 0);
    for (int n = 1; n <= E; ++n) {
        int q1 = (b.en(1, n) == b.en(4, n)) ? 3 : 4;
        for (int q = 1; q <= q1; ++q) ne_num[b.en(q, n)]++;
    }
    int kmax = 0;
    for (int n = 1; n <= N; ++n) kmax = std::max(kmax, ne_num[n]);
    std::vector<int> ne_pos((size_t)kmax * (N + 1), 0);
    auto NEP = [&](int k, int n) -> int & { return ne_pos[(size_t)(n) * kmax + (k - 1)]; };
    std::fill(ne_num.begin(), ne_num.end(), 0);
    for (int n = 1; n <= E; ++n) {
        int q1 = (b.en(1, n) == b.en(4, n)) ? 3 : 4;
        for (int q = 1; q <= q1; ++q) {
            int nd = b.en(q, n);
            ne_num[nd]++;
            NEP(ne_num[nd], nd) = n;
        }
    }
    // neighbour nodes (second pass of the reference, which also fills nn_pos)
    std::vector<int> aux1(N + 1, 0), temp(256);
    std::vector<int> nn_num(N + 1, 0);
    std::vector<std::vector<int>> nn_pos(N + 1);
    for (int n = 1; n <= N; ++n) {
        int counter = 0;
        for (int k = 1; k <= ne_num[n]; ++k) {
            int elem = NEP(k, n);
            int el[4] = {b.en(1, elem), b.en(2, elem), b.en(3, elem), b.en(4, elem)};
            if (el[0] == el[3]) {
                for (int q = 0; q < 3; ++q) {
                    if (el[q] == n) continue;
                    if (aux1[el[q]] != 1) {
                        aux1[el[q]] = 1;
                        temp[counter++] = el[q];
                    }
                }
            } else {
                int ed0 = 0, ed1 = 0;
                if (el[0] == n) { ed0 = el[1]; ed1 = el[3]; }
                if (el[1] == n) { ed0 = el[0]; ed1 = el[2]; }
                if (el[2] == n) { ed0 = el[1]; ed1 = el[3]; }
                if (el[3] == n) { ed0 = el[0]; ed1 = el[2]; }
                int edq[2] = {ed0, ed1};
                for (int q = 0; q < 2; ++q) {
                    if (aux1[edq[q]] != 1) {
                        aux1[edq[q]] = 1;
                        temp[counter++] = edq[q];
                    }
                }
            }
        }
        nn_num[n] = counter + 1;
        for (int i = 0; i < counter; ++i) aux1[temp[i]] = 0;
        nn_pos[n].resize(counter + 1);
        nn_pos[n][0] = n;
        for (int i = 0; i < counter; ++i) nn_pos[n][i + 1] = temp[i];
    }
    // (b) count edges, then internal edges first, boundary edges after
    int counter = 0;
    for (int n = 1; n <= N; ++n)
        for (int q = 2; q <= nn_num[n]; ++q)
            if (nn_pos[n][q - 1] >= n) counter++;
    b.edge2D = counter;
    b.edge_nodes.assign(2 * (size_t)counter, 0);
    b.edge_tri.assign(2 * (size_t)counter, 0);
    int counter_in = 0;
    for (int pass = 0; pass < 2; ++pass) {
        for (int n = 1; n <= N; ++n) {
            for (int q = 2; q <= nn_num[n]; ++q) {
                int node = nn_pos[n][q - 1];
                if (node < n) continue;
                int flag = 0, elems[2] = {0, 0};
                for (int k = 1; k <= ne_num[n]; ++k) {
                    int elem = NEP(k, n);
                    int q2 = (b.en(1, elem) == b.en(4, elem)) ? 3 : 4;
                    for (int q1 = 1; q1 <= q2; ++q1) {
                        if (b.en(q1, elem) == node) {
                            if (flag < 2) elems[flag] = elem;
                            flag++;
                            break;
                        }
                    }
                }
                if ((pass == 0 && flag == 2) || (pass == 1 && flag == 1)) {
                    counter_in++;
                    b.edge_nodes[2 * (counter_in - 1)] = n;
                    b.edge_nodes[2 * (counter_in - 1) + 1] = node;
                    b.edge_tri[2 * (counter_in - 1)] = elems[0];
                    b.edge_tri[2 * (counter_in - 1) + 1] = (pass == 0) ? elems[1] : -999;
                }
            }
        }
        if (pass == 0) b.edge2D_in = counter_in;
    }
    // (d) first element to the left of the edge vector
    for (int n = 1; n <= b.edge2D; ++n) {
        int ed0 = b.edge_nodes[2 * (n - 1)], ed1 = b.edge_nodes[2 * (n - 1) + 1];
        int elem = b.edge_tri[2 * (n - 1)];
        double xc0, xc1, amin;
        b.elem_center(elem, xc0, xc1, amin);
        xc0 = xc0 - b.cx(ed0);
        xc1 = xc1 - b.cy(ed0);
        double xe0 = b.cx(ed1) - b.cx(ed0), xe1 = b.cy(ed1) - b.cy(ed0);
        xe0 = b.cfix(xe0);
        xc0 = b.cfix(xc0);
        if (xc0 * xe1 - xc1 * xe0 > 0.0) {
            int e1 = b.edge_tri[2 * (n - 1)], e2 = b.edge_tri[2 * (n - 1) + 1];
            if (e2 > 0) {
                b.edge_tri[2 * (n - 1)] = e2;
                b.edge_tri[2 * (n - 1) + 1] = e1;
            } else {
                b.edge_nodes[2 * (n - 1) + 1] = ed0;
                b.edge_nodes[2 * (n - 1)] = ed1;
            }
        }
    }
    // (e) elem_edges in the rotation sense of the nodes
    b.elem_edges.assign(4 * (size_t)E, 0);
    std::vector<int> cnt(E + 1, 0);
    for (int n = 1; n <= b.edge2D; ++n)
        for (int k = 0; k < 2; ++k) {
            int q = b.edge_tri[2 * (n - 1) + k];
            if (q > 0) {
                cnt[q]++;
                if (cnt[q] <= 4) b.elem_edges[4 * (q - 1) + cnt[q] - 1] = n;
            }
        }
    auto EN = [&](int k, int e) { return b.edge_nodes[2 * (e - 1) + (k - 1)]; };
    for (int elem = 1; elem <= E; ++elem) {
        int el[4] = {b.en(1, elem), b.en(2, elem), b.en(3, elem), b.en(4, elem)};
        int q1 = (el[0] == el[3]) ? 3 : 4;
        int eled[4];
        for (int k = 0; k < 4; ++k) eled[k] = b.elem_edges[4 * (elem - 1) + k];
        for (int q = 1; q <= q1 - 1; ++q)
            for (int k = 1; k <= q1; ++k) {
                int e = eled[k - 1];
                if (e <= 0) continue;
                if ((EN(1, e) == el[q - 1] && EN(2, e) == el[q]) ||
                    (EN(1, e) == el[q] && EN(2, e) == el[q - 1])) {
                    b.elem_edges[4 * (elem - 1) + q - 1] = e;
                    break;
                }
            }
        for (int k = 1; k <= q1; ++k) {
            int e = eled[k - 1];
            if (e <= 0) continue;
            if ((EN(1, e) == el[q1 - 1] && EN(2, e) == el[0]) ||
                (EN(1, e) == el[0] && EN(2, e) == el[q1 - 1])) {
                b.elem_edges[4 * (elem - 1) + q1 - 1] = e;
                break;
            }
        }
        if (q1 == 3) b.elem_edges[4 * (elem - 1) + 3] = b.elem_edges[4 * (elem - 1)];
    }
}

void find_elem_neighbors(fesomc_mesh_builder &b) {
    const int N = b.nod2D, E = b.elem2D;
    b.elem_neighbors.assign(4 * (size_t)E, 0);
    for (int elem = 1; elem <= E; ++elem) {
        const int32_t *eled = &b.elem_edges[4 * (elem - 1)];
        int q = 4;
        if (eled[0] == eled[3] || eled[3] == 0) q = 3;
        for (int j = 1; j <= q; ++j) {
            int e = eled[j - 1];
            int elem1 = b.edge_tri[2 * (e - 1)];
            if (elem1 == elem) elem1 = b.edge_tri[2 * (e - 1) + 1];
            b.elem_neighbors[4 * (elem - 1) + j - 1] = elem1;
        }
        if (q == 3) b.elem_neighbors[4 * (elem - 1) + 3] = b.elem_neighbors[4 * (elem - 1)];
    }
    b.nod_in_elem2D_num.assign(N, 0);
    for (int el = 1; el <= E; ++el) {
        int q = (b.en(1, el) == b.en(4, el)) ? 3 : 4;
        for (int j = 1; j <= q; ++j) b.nod_in_elem2D_num[b.en(j, el) - 1]++;
    }
    int mx = 0;
    for (int n = 0; n < N; ++n) mx = std::max(mx, (int)b.nod_in_elem2D_num[n]);
    b.nie_max = mx;
    b.nod_in_elem2D.assign((size_t)mx * N, 0);
    std::fill(b.nod_in_elem2D_num.begin(), b.nod_in_elem2D_num.end(), 0);
    for (int el = 1; el <= E; ++el) {
        int q = (b.en(1, el) == b.en(4, el)) ? 3 : 4;
        for (int j = 1; j <= q; ++j) {
            int nd = b.en(j, el);
            int k = ++b.nod_in_elem2D_num[nd - 1];
            b.nod_in_elem2D[(size_t)mx * (nd - 1) + k - 1] = el;
        }
    }
}

void mesh_arrays1(fesomc_mesh_builder &b, int coriolis_on, double lat_cartesian) {
    const int N = b.nod2D, E = b.elem2D;
    b.elem_area.assign(E, 0.0);
    b.elem_cos.assign(E, 0.0);
    b.area.assign(N, 0.0);
    b.metric_factor.assign(E, 0.0);
    b.coriolis.assign(E, 0.0);
    b.w_cv.assign(4 * (size_t)E, 0.0);
    for (int elem = 1; elem <= E; ++elem) {
        double ax, ay, aa;
        b.elem_center(elem, ax, ay, aa);
        b.coriolis[elem - 1] = 2.0 * kOmega * std::sin(ay);
        b.elem_cos[elem - 1] = std::cos(ay);
        b.metric_factor[elem - 1] = std::tan(ay) / kREarth;
        b.elem_area[elem - 1] = aa;
    }
    if (b.cartesian) {
        for (int e = 0; e < E; ++e) { b.elem_cos[e] = 1.0; b.metric_factor[e] = 0.0; }
    }
    if (coriolis_on) {
        if (b.cartesian)
            for (int e = 0; e < E; ++e) b.coriolis[e] = 2.0 * kOmega * std::sin(lat_cartesian);
    } else {
        for (int e = 0; e < E; ++e) b.coriolis[e] = 0.0;
    }
    for (int e = 0; e < E; ++e) b.elem_area[e] = b.elem_area[e] * b.elem_cos[e];

    for (int elem = 1; elem <= E; ++elem) {
        int eln[6];
        for (int j = 2; j <= 5; ++j) eln[j - 1] = b.en(j - 1, elem);
        if (eln[1] == eln[4]) {
            for (int j = 2; j <= 4; ++j) {
                b.area[eln[j - 1] - 1] = b.area[eln[j - 1] - 1] + b.elem_area[elem - 1] / 3.0;
                b.w_cv[4 * (elem - 1) + j - 2] = 1.0 / 3.0;
            }
        } else {
            double rc0, rc1, aa;
            b.elem_center(elem, rc0, rc1, aa);
            eln[0] = eln[4];
            eln[5] = eln[1];
            for (int j = 2; j <= 5; ++j) {
                double r10 = b.cx(eln[j - 2]), r11 = b.cy(eln[j - 2]);
                double r00 = b.cx(eln[j - 1]), r01 = b.cy(eln[j - 1]);
                double rr0 = b.cfix(r10 - r00), rr1 = r11 - r01;
                r10 = b.cx(eln[j]);
                r11 = b.cy(eln[j]);
                double rl0 = b.cfix(r10 - r00), rl1 = r11 - r01;
                double q0 = b.cfix(rc0 - r00), q1 = rc1 - r01;
                double part = 0.25 * b.elem_cos[elem - 1] *
                              (std::fabs(rl0 * q1 - rl1 * q0) + std::fabs(rr0 * q1 - rr1 * q0));
                b.area[eln[j - 1] - 1] = b.area[eln[j - 1] - 1] + part;
                b.w_cv[4 * (elem - 1) + j - 2] = part / b.elem_area[elem - 1];
            }
        }
    }
    for (int e = 0; e < E; ++e) b.elem_area[e] = b.elem_area[e] * kREarth * kREarth;
    for (int n = 0; n < N; ++n) b.area[n] = b.area[n] * kREarth * kREarth;
}

void mesh_arrays2(fesomc_mesh_builder &b) {
    const int E = b.elem2D, Ed = b.edge2D;
    b.edge_dxdy.assign(2 * (size_t)Ed, 0.0);
    b.edge_cross_dxdy.assign(4 * (size_t)Ed, 0.0);
    b.gradient_sca.assign(8 * (size_t)E, 0.0);
    b.gradient_vec.assign(8 * (size_t)E, 0.0);
    b.center_x.assign(E, 0.0);
    b.center_y.assign(E, 0.0);
    for (int n = 1; n <= E; ++n) {
        double ax, ay, aa;
        b.elem_center(n, ax, ay, aa);
        b.center_x[n - 1] = ax;
        b.center_y[n - 1] = ay;
    }
    for (int n = 1; n <= Ed; ++n) {
        int e0 = b.edge_nodes[2 * (n - 1)], e1 = b.edge_nodes[2 * (n - 1) + 1];
        double a0 = b.cx(e1) - b.cx(e0), a1 = b.cy(e1) - b.cy(e0);
        a0 = b.cfix(a0);
        b.edge_dxdy[2 * (n - 1)] = a0;
        b.edge_dxdy[2 * (n - 1) + 1] = a1;
    }
    for (int edg = 1; edg <= Ed; ++edg) {
        int e0 = b.edge_nodes[2 * (edg - 1)], e1 = b.edge_nodes[2 * (edg - 1) + 1];
        int el1 = b.edge_tri[2 * (edg - 1)], el2 = b.edge_tri[2 * (edg - 1) + 1];
        double a0, a1;
        b.edge_center(e0, e1, a0, a1);
        double b0 = b.center_x[el1 - 1] - a0, b1 = b.center_y[el1 - 1] - a1;
        b0 = b.cfix(b0);
        b0 = b0 * b.elem_cos[el1 - 1];
        b0 = b0 * kREarth;
        b1 = b1 * kREarth;
        b.edge_cross_dxdy[4 * (edg - 1)] = b0;
        b.edge_cross_dxdy[4 * (edg - 1) + 1] = b1;
        if (el2 > 0) {
            b0 = b.center_x[el2 - 1] - a0;
            b1 = b.center_y[el2 - 1] - a1;
            b0 = b.cfix(b0);
            b0 = b0 * b.elem_cos[el2 - 1];
            b0 = b0 * kREarth;
            b1 = b1 * kREarth;
            b.edge_cross_dxdy[4 * (edg - 1) + 2] = b0;
            b.edge_cross_dxdy[4 * (edg - 1) + 3] = b1;
        }
    }
    for (int elem = 1; elem <= E; ++elem) {
        double *gs = &b.gradient_sca[8 * (elem - 1)];
        int el[4] = {b.en(1, elem), b.en(2, elem), b.en(3, elem), b.en(4, elem)};
        double ec = b.elem_cos[elem - 1];
        if (el[0] == el[3]) {
            double dX31 = b.cfix(b.cx(el[2]) - b.cx(el[0]));
            dX31 = ec * dX31;
            double dX21 = b.cfix(b.cx(el[1]) - b.cx(el[0]));
            dX21 = ec * dX21;
            double dY31 = b.cy(el[2]) - b.cy(el[0]);
            double dY21 = b.cy(el[1]) - b.cy(el[0]);
            double dfactor = (-0.5 * kREarth) / b.elem_area[elem - 1];
            gs[0] = (-dY31 + dY21) * dfactor;
            gs[1] = dY31 * dfactor;
            gs[2] = -dY21 * dfactor;
            gs[3] = 0.0;
            gs[4] = (dX31 - dX21) * dfactor;
            gs[5] = -dX31 * dfactor;
            gs[6] = dX21 * dfactor;
            gs[7] = 0.0;
        } else {
            int enodes[6] = {el[3], el[0], el[1], el[2], el[3], el[0]};
            double dfactor = (0.5 * kREarth) / b.elem_area[elem - 1];
            for (int j = 2; j <= 5; ++j) {
                double x10 = b.cx(enodes[j - 1]), x11 = b.cy(enodes[j - 1]);
                double x20 = b.cx(enodes[j - 2]), x21 = b.cy(enodes[j - 2]);
                double xd0 = b.cfix(x10 - x20), xd1 = x11 - x21;
                x20 = b.cx(enodes[j]);
                x21 = b.cy(enodes[j]);
                double y0 = b.cfix(x20 - x10), y1 = x21 - x11;
                xd0 = xd0 + y0;
                xd1 = xd1 + y1;
                xd0 = xd0 * ec;
                gs[j - 2] = -xd1 * dfactor;
                gs[j - 2 + 4] = xd0 * dfactor;
            }
        }
    }
    for (int elem = 1; elem <= E; ++elem) {
        double a0 = b.center_x[elem - 1], a1 = b.center_y[elem - 1];
        int q = (b.en(1, elem) == b.en(4, elem)) ? 3 : 4;
        double x[4] = {0, 0, 0, 0}, y[4] = {0, 0, 0, 0};
        for (int j = 1; j <= q; ++j) {
            int e1 = b.elem_neighbors[4 * (elem - 1) + j - 1];
            if (e1 > 0) {
                x[j - 1] = b.cfix(b.center_x[e1 - 1] - a0);
                y[j - 1] = b.center_y[e1 - 1] - a1;
            } else {
                int ed = b.elem_edges[4 * (elem - 1) + j - 1];
                double bb0, bb1;
                b.edge_center(b.edge_nodes[2 * (ed - 1)], b.edge_nodes[2 * (ed - 1) + 1], bb0, bb1);
                x[j - 1] = b.cfix(bb0 - a0);
                x[j - 1] = 2.0 * x[j - 1];
                y[j - 1] = 2.0 * (bb1 - a1);
            }
        }
        if (q == 3) { x[3] = 0.0; y[3] = 0.0; }
        for (int j = 0; j < 4; ++j) {
            x[j] = x[j] * b.elem_cos[elem - 1] * kREarth;
            y[j] = y[j] * kREarth;
        }
        double cxx = 0.0, cxy = 0.0, cyy = 0.0;
        for (int j = 0; j < 4; ++j) cxx = cxx + x[j] * x[j];
        for (int j = 0; j < 4; ++j) cxy = cxy + x[j] * y[j];
        for (int j = 0; j < 4; ++j) cyy = cyy + y[j] * y[j];
        double d = cxy * cxy - cxx * cyy;
        double *gv = &b.gradient_vec[8 * (elem - 1)];
        for (int j = 0; j < 4; ++j) {
            gv[j] = (cxy * y[j] - cyy * x[j]) / d;
            gv[j + 4] = (cxy * x[j] - cxx * y[j]) / d;
        }
    }
}

// find_up_downwind_triangles.  Inside the element loop the reference uses
// CYCLE after a match, so the last matching element wins.
void find_up_dn(fesomc_mesh_builder &b) {
    const int Ed = b.edge2D;
    b.edge_up_dn_tri.assign(2 * (size_t)Ed, 0);
    auto ce = [&](int k, int q, int elem) {  // coord_elem(k,q,elem)
        int nd = b.en(q, elem);
        return k == 1 ? b.cx(nd) : b.cy(nd);
    };
    for (int n = 1; n <= Ed; ++n) {
        int ed[2] = {b.edge_nodes[2 * (n - 1)], b.edge_nodes[2 * (n - 1) + 1]};
        double x0 = b.cx(ed[1]) - b.cx(ed[0]), x1 = b.cy(ed[1]) - b.cy(ed[0]);
        x0 = b.cfix(x0);
        for (int side = 0; side < 2; ++side) {
            x0 = -x0;
            x1 = -x1;
            int nd = ed[side];
            for (int k = 1; k <= b.nod_in_elem2D_num[nd - 1]; ++k) {
                int elem = b.nod_in_elem2D[(size_t)b.nie_max * (nd - 1) + k - 1];
                bool tri = b.en(1, elem) == b.en(4, elem);
                int ib, ic, io;  // b = node ib - node io, c = node ic - node io
                if (tri) {
                    if (b.en(1, elem) == nd) { io = 1; ib = 2; ic = 3; }
                    else if (b.en(2, elem) == nd) { io = 2; ib = 1; ic = 3; }
                    else { io = 3; ib = 1; ic = 2; }
                } else {
                    if (b.en(1, elem) == nd) { io = 1; ib = 2; ic = 4; }
                    else if (b.en(2, elem) == nd) { io = 2; ib = 3; ic = 1; }
                    else if (b.en(3, elem) == nd) { io = 3; ib = 4; ic = 2; }
                    else { io = 4; ib = 1; ic = 3; }
                }
                double b0 = ce(1, ib, elem) - ce(1, io, elem), b1 = ce(2, ib, elem) - ce(2, io, elem);
                double c0 = ce(1, ic, elem) - ce(1, io, elem), c1 = ce(2, ic, elem) - ce(2, io, elem);
                b0 = b.cfix(b0);
                c0 = b.cfix(c0);
                double cr = c0 * c0 + c1 * c1;
                double bx = (b0 * c0 + b1 * c1) / cr;
                double by = (-b0 * c1 + b1 * c0) / cr;
                double xx = (x0 * c0 + x1 * c1) / cr;
                double xy = (-x0 * c1 + x1 * c0) / cr;
                double ab = std::atan2(by, bx);
                double ax = std::atan2(xy, xx);
                bool hit = (ab > 0 && ax > 0 && ax < ab) || (ab < 0 && ax < 0 && ax > ab) ||
                           (ab == ax) || (ax == 0.0);
                if (hit) b.edge_up_dn_tri[2 * (n - 1) + side] = elem;
            }
        }
    }
    b.have_up_dn = true;
}

void set_sigma(fesomc_mesh_builder &b, const fesomc_mesh_opts &o) {
    const int ns = o.nsigma;
    b.sigma.assign(ns, 0.0);
    if (o.ind_sigma == 2) {
        for (int K = 1; K <= ns; ++K) {
            double X1 = std::tanh((o.lev_bot + o.lev_sur) * (ns - K) / (ns - 1) - o.lev_bot);
            double X2 = std::tanh(o.lev_bot);
            double X3 = X2 + std::tanh(o.lev_sur);
            b.sigma[K - 1] = (X1 + X2) / X3;
        }
    } else if (o.pow_sig == 1.0) {
        for (int K = 1; K <= ns; ++K)
            b.sigma[K - 1] = -std::pow((K - 1) / (double)(ns - 1), o.pow_sig) + 1.0;
    } else {
        int h = (ns + 1) / 2;
        for (int K = 1; K <= h; ++K)
            b.sigma[K - 1] = -(std::pow((K - 1) / (double)(h - 1), o.pow_sig) * 0.5) + 1.0;
        for (int K = h + 1; K <= ns; ++K)
            b.sigma[K - 1] = std::pow((ns - K) / (double)(h - 1), o.pow_sig) * 0.5;
    }
}

}  // namespace

extern "C" int fesomc_mesh_build(int32_t nod2D, const double *xy, const int32_t *index_nod2D,
                                 int32_t elem2D, const int32_t *elem_nodes4,
                                 const double *depth, const fesomc_mesh_opts *opts,
                                 fesomc_mesh_builder **out) {
    if (!out || !xy || !index_nod2D || !elem_nodes4 || !depth || !opts) return FESOMC_EINVAL;
    if (nod2D <= 2 || elem2D <= 0 || opts->nsigma < 3) return FESOMC_EINVAL;
    if (opts->ind_sigma != 1 && opts->ind_sigma != 2) return FESOMC_EINVAL;
    *out = nullptr;
    fesomc_mesh_builder *b = new (std::nothrow) fesomc_mesh_builder();
    if (!b) return FESOMC_ENOMEM;
    b->nod2D = nod2D;
    b->elem2D = elem2D;
    b->nsigma = opts->nsigma;
    b->cartesian = opts->cartesian != 0;
    b->cyclic_length = opts->cyclic_length_deg * kRad;
    b->coord.resize(2 * (size_t)nod2D);
    b->index_nod2D.assign(index_nod2D, index_nod2D + nod2D);
    for (int n = 0; n < nod2D; ++n) {
        if (b->cartesian) {
            b->coord[2 * n] = xy[2 * n] / kREarth;
            b->coord[2 * n + 1] = xy[2 * n + 1] / kREarth;
        } else {
            b->coord[2 * n] = xy[2 * n] * kRad;
            b->coord[2 * n + 1] = xy[2 * n + 1] * kRad;
        }
        if (b->index_nod2D[n] == 2) b->in_obn.push_back(n + 1);
    }
    // triangles first, then quads, each in file order (fv_main.F90:866-883)
    b->elem2D_nodes.resize(4 * (size_t)elem2D);
    int ntri = 0;
    for (int n = 0; n < elem2D; ++n) {
        const int32_t *nd = elem_nodes4 + 4 * n;
        for (int q = 0; q < 4; ++q)
            if (nd[q] < 1 || nd[q] > nod2D) { delete b; return FESOMC_EINVAL; }
        if (nd[0] == nd[3]) { std::memcpy(&b->elem2D_nodes[4 * (size_t)ntri], nd, 16); ntri++; }
    }
    int nq = 0;
    for (int n = 0; n < elem2D; ++n) {
        const int32_t *nd = elem_nodes4 + 4 * n;
        if (nd[0] != nd[3]) { std::memcpy(&b->elem2D_nodes[4 * (size_t)(ntri + nq)], nd, 16); nq++; }
    }
    b->elem2D_tri = ntri;
    b->depth.assign(depth, depth + nod2D);
    int rc = test_elem(*b);
    if (rc) { delete b; return rc; }
    find_edges(*b);
    find_elem_neighbors(*b);
    mesh_arrays1(*b, opts->coriolis_on, opts->lat_cartesian_deg * kPi / 180.0);
    mesh_arrays2(*b);
    set_sigma(*b, *opts);
    if (opts->with_up_dn_tri) find_up_dn(*b);
    b->a_tp.assign(2 * (size_t)nod2D, 0.0);
    for (int n = 0; n < nod2D; ++n) {
        double a1 = opts->T_potential ? 0.918 : 1.0, a2 = opts->T_potential ? 0.69 : 0.0;
        if (b->index_nod2D[n] == 2) { a1 = 1.0; a2 = 0.0; }
        b->a_tp[n] = a1;
        b->a_tp[nod2D + n] = a2;
    }
    b->ac.assign(nod2D, 1.0);
    *out = b;
    return FESOMC_OK;
}

extern "C" int fesomc_mesh_view(const fesomc_mesh_builder *b, fesomc_mesh *m) {
    if (!b || !m) return FESOMC_EINVAL;
    std::memset(m, 0, sizeof(*m));
    m->nod2D = b->nod2D;
    m->elem2D = b->elem2D;
    m->edge2D = b->edge2D;
    m->edge2D_in = b->edge2D_in;
    m->nsigma = b->nsigma;
    m->nod_in_elem2D_max = b->nie_max;
    m->index_nod2D = b->index_nod2D.data();
    m->elem2D_nodes = b->elem2D_nodes.data();
    m->edge_nodes = b->edge_nodes.data();
    m->edge_tri = b->edge_tri.data();
    m->elem_edges = b->elem_edges.data();
    m->elem_neighbors = b->elem_neighbors.data();
    m->nod_in_elem2D_num = b->nod_in_elem2D_num.data();
    m->nod_in_elem2D = b->nod_in_elem2D.data();
    m->edge_up_dn_tri = b->have_up_dn ? b->edge_up_dn_tri.data() : nullptr;
    m->coord_nod2D = b->coord.data();
    m->depth = b->depth.data();
    m->area = b->area.data();
    m->elem_area = b->elem_area.data();
    m->elem_cos = b->elem_cos.data();
    m->coriolis = b->coriolis.data();
    m->w_cv = b->w_cv.data();
    m->gradient_sca = b->gradient_sca.data();
    m->gradient_vec = b->gradient_vec.data();
    m->edge_dxdy = b->edge_dxdy.data();
    m->edge_cross_dxdy = b->edge_cross_dxdy.data();
    m->sigma = b->sigma.data();
    m->a_tp = b->a_tp.data();
    m->ac = b->ac.data();
    m->nobn = (int32_t)b->in_obn.size();
    m->in_obn = b->in_obn.empty() ? nullptr : b->in_obn.data();
    m->n_rivers = (int32_t)b->nod_rivers.size();
    m->nod_rivers = b->nod_rivers.empty() ? nullptr : b->nod_rivers.data();
    return FESOMC_OK;
}

extern "C" double fesomc_mesh_scale_area(const fesomc_mesh_builder *b) {
    if (!b) return 0.0;
    double s = 0.0;
    for (double a : b->elem_area) s = s + a;
    return s / b->elem2D;
}

extern "C" int fesomc_mesh_set_rivers(fesomc_mesh_builder *b, int32_t n, const int32_t *nodes) {
    if (!b || n < 0 || (n > 0 && !nodes)) return FESOMC_EINVAL;
    for (int i = 0; i < n; ++i)
        if (nodes[i] < 1 || nodes[i] > b->nod2D) return FESOMC_EINVAL;
    b->nod_rivers.assign(nodes, nodes + n);
    return FESOMC_OK;
}

// Sponge layer at the open boundary (ac_create_Xobn / ac_create /
// Dist2in1, src/fv_utilit.F90:53-88,151-220): ac = distance to the nearest
// open-boundary node / radius inside the radius, 1 elsewhere.  Open-boundary
// nodes are those with index_nod2D = 2, in node order.
extern "C" int fesomc_mesh_set_sponge(fesomc_mesh_builder *b, double radius) {
    if (!b || !(radius > 0.0)) return FESOMC_EINVAL;
    std::vector<double> x1, x2;
    for (int n = 1; n <= b->nod2D; ++n)
        if (b->index_nod2D[n - 1] == 2) {
            x1.push_back(b->cx(n));
            x2.push_back(b->cy(n));
        }
    b->ac.assign(b->nod2D, 1.0);
    if (x1.empty()) return FESOMC_OK;
    const size_t nob = x1.size();
    for (int n = 1; n <= b->nod2D; ++n) {
        const double X1 = b->cx(n), X2 = b->cy(n);
        double d2obn;
        if (b->cartesian) {
            double d = (x1[0] - X1) * (x1[0] - X1) + (x2[0] - X2) * (x2[0] - X2);
            for (size_t j = 1; j < nob; ++j) {
                const double t = (x1[j] - X1) * (x1[j] - X1) + (x2[j] - X2) * (x2[j] - X2);
                if (t < d) d = t;
            }
            d2obn = std::sqrt(d) * kREarth;
        } else {
            const double cos_X2 = std::cos(X2);
            auto hav = [&](size_t j) {
                const double s2 = std::sin((x2[j] - X2) * 0.5), s1 = std::sin((x1[j] - X1) * 0.5);
                // Fortran precedence: cos_X2 * cos(X2obn) * sin(..)**2 is (cos_X2 * cos) * (s1 * s1)
                return s2 * s2 + cos_X2 * std::cos(x2[j]) * (s1 * s1);
            };
            double a = hav(0);
            for (size_t j = 1; j < nob; ++j) {
                const double t = hav(j);
                if (t < a) a = t;
            }
            d2obn = 2.0 * kREarth * std::asin(std::min(1.0, std::sqrt(a)));
        }
        if (d2obn < radius) b->ac[n - 1] = d2obn / radius;
    }
    return FESOMC_OK;
}

extern "C" void fesomc_mesh_free(fesomc_mesh_builder *b) { delete b; }

// densityJM (src/fv_pressure_new.F90:340-414) for host-side initialisation.
// Literals written without _WP in the reference are REAL(4) constants.
namespace {
inline double r4(float x) { return static_cast<double>(x); }
}  // namespace

extern "C" double fesomc_host_density_jm(double t, double s, double pz, double density_0) {
    double ss3 = std::sqrt(s * s * s);
    double bulk = 19092.56 + t * (209.8925 - t * (3.041638 - t * (-r4(1.852732e-3f) - t * (r4(1.361629e-5f)))))
                + s * (104.4077 - t * (6.500517 - t * (.1553190 - t * (-r4(2.326469e-4f)))))
                + ss3 * (-5.587545 + t * (0.7390729 - t * (r4(1.909078e-2f))))
                - pz * (r4(4.721788e-1f) + t * (r4(1.028859e-2f) + t * (-r4(2.512549e-4f) - t * (r4(5.939910e-7f)))))
                - pz * s * (-r4(1.571896e-2f) - t * (r4(2.598241e-4f) + t * (-r4(7.267926e-6f))))
                - pz * ss3 * r4(2.042967e-3f)
                + pz * pz * (r4(1.045941e-5f) - t * (r4(5.782165e-10f) - t * (r4(1.296821e-7f))))
                + pz * pz * s * (-r4(2.595994e-7f) + t * (-r4(1.248266e-9f) + t * (-r4(3.508914e-9f))));
    double rhopot = 999.842594
                  + t * (r4(6.793952e-2f) + t * (-r4(9.095290e-3f) + t * (r4(1.001685e-4f)
                  + t * (-r4(1.120083e-6f) + t * r4(6.536332e-9f)))))
                  + s * (0.824493 + t * (-r4(4.08990e-3f) + t * (r4(7.64380e-5f)
                  + t * (-r4(8.24670e-7f) + t * r4(5.38750e-9f)))))
                  + ss3 * (-r4(5.72466e-3f) + t * (r4(1.02270e-4f) + t * (-r4(1.65460e-6f))))
                  + r4(4.8314e-4f) * s * s;
    return rhopot * bulk / (bulk + 0.1 * pz) - density_0;
}
