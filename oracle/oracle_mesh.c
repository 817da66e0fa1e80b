/*
 * oracle_mesh.c -- CPU restatement of the reference's mesh set-up, part of
 * the oracle (test infrastructure only: loaded by tests/, the smoke check and
 * bench.py's CPU legs, never by the GPU product path).
 *
 * It is written from the Fortran alone, independently of the product's host
 * mesh builder, so that the two can be checked against each other array by
 * array and so that the oracle (and bench.py's reference arm) builds its
 * meshes without loading the product library.  Each routine follows one
 * reference routine, statement by statement, with the operand order of every
 * floating-point expression kept (built with -ffp-contract=off):
 *
 *   read_mesh_ser               src/fv_main.F90:787-945 (coordinate scaling,
 *                               triangles first, open-boundary list)
 *   test_elem                   src/fv_mesh_array.F90:1-82
 *   find_edges                  src/fv_mesh_array.F90:395-718
 *   edge_center / elem_center   src/fv_mesh_array.F90:720-789
 *   find_elem_neighbors         src/fv_mesh_array.F90:791-946 (serial part)
 *   mesh_arrays1 / cdiff        src/fv_mesh_array.F90:948-1152
 *   mesh_arrays2                src/fv_mesh_array.F90:1155-1386
 *   find_up_downwind_triangles  src/fv_mesh_array.F90:1390-1618
 *   SET_SIGMA cases 1, 2        src/fv_vert_coord.F90:135-200
 *   scale_area, a_tp            src/fv_ini.F90:81,94-107
 *   ac_create / Dist2in1        src/fv_utilit.F90:53-88,150-220, set-up
 *                               src/fv_main.F90:224-250
 *
 * Arrays are kept 1-based in the Fortran layout (column-major, first index
 * fastest), the layout fesomc_mesh hands to the library.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../include/fesomc_gpu.h"

#define O_PI 3.14159265358979                    /* fv_var.F90:8, as written */
#define O_RAD (O_PI / 180.0)                     /* fv_var.F90:9 */
#define O_REARTH 6400000.0                       /* fv_var.F90:14 */

typedef struct oracle_mesh {
    int N, E, Ed, Ed_in, NS, nie_max, cart;
    double cyc;                                  /* cyclic_length (radians) */
    int32_t *index, *en, *edge_nodes, *edge_tri, *elem_edges, *elem_nb, *nie_num, *nie, *updn, *in_obn, *rivers;
    int nobn, nriv;
    double *coord, *depth, *area, *elem_area, *elem_cos, *coriolis, *w_cv, *gs, *gv, *edxdy, *ecross, *sigma,
        *a_tp, *ac, *cx, *cy;
} oracle_mesh;

/* 1-based accessors in the Fortran layout */
#define EN(m, q, e) ((m)->en[4 * ((e)-1) + (q)-1])
#define CX(m, n) ((m)->coord[2 * ((n)-1)])
#define CY(m, n) ((m)->coord[2 * ((n)-1) + 1])
#define ED(m, k, e) ((m)->edge_nodes[2 * ((e)-1) + (k)-1])
#define ET(m, k, e) ((m)->edge_tri[2 * ((e)-1) + (k)-1])
#define EE(m, q, e) ((m)->elem_edges[4 * ((e)-1) + (q)-1])

static double cyc_fix(const oracle_mesh *m, double d) {
    if (d > m->cyc / 2.0) d = d - m->cyc;
    if (d < -m->cyc / 2.0) d = d + m->cyc;
    return d;
}

/* edge_center (fv_mesh_array.F90:720-740) */
static void edge_center(const oracle_mesh *m, int n1, int n2, double *x, double *y) {
    double a1 = CX(m, n1), a2 = CY(m, n1), b1 = CX(m, n2), b2 = CY(m, n2);
    if (a1 - b1 > m->cyc / 2.0) a1 = a1 - m->cyc;
    if (a1 - b1 < -m->cyc / 2.0) b1 = b1 - m->cyc;
    *x = 0.5 * (a1 + b1);
    *y = 0.5 * (a2 + b2);
}

/* elem_center (fv_mesh_array.F90:742-789) */
static void elem_center(const oracle_mesh *m, int elem, double *x, double *y, double *s) {
    double ax[4], ay[4];
    for (int k = 0; k < 4; ++k) {
        ax[k] = CX(m, EN(m, k + 1, elem));
        ay[k] = CY(m, EN(m, k + 1, elem));
    }
    if (EN(m, 1, elem) == EN(m, 4, elem)) {
        double amin = ax[0];
        for (int k = 1; k < 3; ++k)
            if (ax[k] < amin) amin = ax[k];
        for (int k = 0; k < 3; ++k)
            if (ax[k] - amin > m->cyc / 2.0) ax[k] = ax[k] - m->cyc;
        *x = ((ax[0] + ax[1]) + ax[2]) / 3.0;
        *y = ((ay[0] + ay[1]) + ay[2]) / 3.0;
        *s = 0.5 * fabs((ax[1] - ax[0]) * (ay[2] - ay[0]) - (ay[1] - ay[0]) * (ax[2] - ax[0]));
    } else {
        double amin = ax[0];
        for (int k = 1; k < 4; ++k)
            if (ax[k] < amin) amin = ax[k];
        for (int k = 0; k < 4; ++k)
            if (ax[k] - amin > m->cyc / 2.0) ax[k] = ax[k] - m->cyc;
        double xx = ax[0] + ax[2] + ax[3];
        double yy = ay[0] + ay[2] + ay[3];
        double x1 = ax[0] + ax[1] + ax[2];
        double y1 = ay[0] + ay[1] + ay[2];
        double s1 = fabs((ax[2] - ax[3]) * (ay[0] - ay[3]) - (ay[2] - ay[3]) * (ax[0] - ax[3]));
        double s2 = fabs((ax[2] - ax[1]) * (ay[0] - ay[1]) - (ay[2] - ay[1]) * (ax[0] - ax[1]));
        *x = (xx * s1 + x1 * s2) / 3.0 / (s1 + s2);
        *y = (yy * s1 + y1 * s2) / 3.0 / (s1 + s2);
        *s = 0.5 * (s1 + s2);
    }
}

/* test_elem (fv_mesh_array.F90:1-82): clockwise node order, or the
 * "Node list problem" stop for a self-crossing quad */
static int test_elem(oracle_mesh *m) {
    for (int n = 1; n <= m->E; ++n) {
        int32_t *el = &m->en[4 * (n - 1)];
        double a1 = CX(m, el[0]), a2 = CY(m, el[0]);
        double b1 = CX(m, el[1]) - a1, b2 = CY(m, el[1]) - a2;
        double c1 = CX(m, el[2]) - a1, c2 = CY(m, el[2]) - a2;
        b1 = cyc_fix(m, b1);
        c1 = cyc_fix(m, c1);
        if (el[0] == el[3]) {
            double r = b1 * c2 - b2 * c1;
            if (r > 0.0) {
                int32_t t = el[1];
                el[1] = el[2];
                el[2] = t;
            }
        } else {
            double d1 = CX(m, el[3]) - a1, d2 = CY(m, el[3]) - a2;
            d1 = cyc_fix(m, d1);
            double r = b1 * c2 - b2 * c1;
            double r1 = b1 * d2 - b2 * d1;
            if (r1 * r < 0.0) return FESOMC_EMESH;
            if (r > 0) {
                int32_t t = el[1];
                el[1] = el[3];
                el[3] = t;
            }
        }
    }
    return FESOMC_OK;
}

/* the two neighbours of node n inside quad elem that share an edge with n,
 * as the node-neighbourhood loops of find_edges pick them */
static void quad_edge_nbrs(const oracle_mesh *m, int elem, int n, int *e1, int *e2) {
    int q1 = EN(m, 1, elem), q2 = EN(m, 2, elem), q3 = EN(m, 3, elem), q4 = EN(m, 4, elem);
    if (q1 == n) { *e1 = q2; *e2 = q4; }
    if (q2 == n) { *e1 = q1; *e2 = q3; }
    if (q3 == n) { *e1 = q2; *e2 = q4; }
    if (q4 == n) { *e1 = q1; *e2 = q3; }
}

/* find_edges (fv_mesh_array.F90:395-718) */
static int find_edges(oracle_mesh *m) {
    const int N = m->N, E = m->E;
    int *ne_num = calloc((size_t)N + 1, sizeof(int));
    if (!ne_num) return FESOMC_ENOMEM;
    for (int n = 1; n <= E; ++n) {
        int q1 = (EN(m, 1, n) == EN(m, 4, n)) ? 3 : 4;
        for (int q = 1; q <= q1; ++q) ne_num[EN(m, q, n)]++;
    }
    int kmax = 0;
    for (int n = 1; n <= N; ++n)
        if (ne_num[n] > kmax) kmax = ne_num[n];
    int *ne_pos = malloc(sizeof(int) * (size_t)kmax * (size_t)(N + 1));
    memset(ne_num, 0, sizeof(int) * ((size_t)N + 1));
    for (int n = 1; n <= E; ++n) {
        int q1 = (EN(m, 1, n) == EN(m, 4, n)) ? 3 : 4;
        for (int q = 1; q <= q1; ++q) {
            int nd = EN(m, q, n);
            ne_num[nd]++;
            ne_pos[(size_t)kmax * nd + ne_num[nd] - 1] = n;
        }
    }
    /* neighbouring nodes, first the node itself (nn_pos(1,n) = n) */
    int *aux1 = calloc((size_t)N + 1, sizeof(int));
    int *nn_num = calloc((size_t)N + 1, sizeof(int));
    int nnmax = 2 * kmax + 1;
    int *nn_pos = malloc(sizeof(int) * (size_t)nnmax * (size_t)(N + 1));
    int temp[256];
    for (int n = 1; n <= N; ++n) {
        int counter = 0;
        for (int k = 0; k < ne_num[n]; ++k) {
            int elem = ne_pos[(size_t)kmax * n + k];
            if (EN(m, 1, elem) == EN(m, 4, elem)) {
                for (int q = 1; q <= 3; ++q) {
                    int nd = EN(m, q, elem);
                    if (nd == n) continue;
                    if (aux1[nd] != 1) {
                        aux1[nd] = 1;
                        temp[counter++] = nd;
                    }
                }
            } else {
                int ed[2] = {0, 0};
                quad_edge_nbrs(m, elem, n, &ed[0], &ed[1]);
                for (int q = 0; q < 2; ++q)
                    if (aux1[ed[q]] != 1) {
                        aux1[ed[q]] = 1;
                        temp[counter++] = ed[q];
                    }
            }
        }
        nn_num[n] = counter + 1;
        for (int q = 0; q < counter; ++q) aux1[temp[q]] = 0;
        nn_pos[(size_t)nnmax * n] = n;
        for (int q = 0; q < counter; ++q) nn_pos[(size_t)nnmax * n + 1 + q] = temp[q];
    }
    /* (b) edges: internal ones first, then the boundary ones, each in the
     * discovery order (node n, neighbours with a larger number) */
    int counter = 0;
    for (int n = 1; n <= N; ++n)
        for (int q = 2; q <= nn_num[n]; ++q)
            if (nn_pos[(size_t)nnmax * n + q - 1] >= n) counter++;
    m->Ed = counter;
    m->edge_nodes = malloc(sizeof(int32_t) * 2 * (size_t)counter);
    m->edge_tri = malloc(sizeof(int32_t) * 2 * (size_t)counter);
    int counter_in = 0;
    for (int pass = 0; pass < 2; ++pass) {
        for (int n = 1; n <= N; ++n) {
            for (int q = 2; q <= nn_num[n]; ++q) {
                int node = nn_pos[(size_t)nnmax * n + q - 1];
                if (node < n) continue;
                int flag = 0, elems[2] = {0, 0};
                for (int k = 0; k < ne_num[n]; ++k) {
                    int elem = ne_pos[(size_t)kmax * n + k];
                    int q2 = (EN(m, 1, elem) == EN(m, 4, elem)) ? 3 : 4;
                    for (int qq = 1; qq <= q2; ++qq)
                        if (EN(m, qq, elem) == node) {
                            if (flag < 2) elems[flag] = elem;
                            flag++;
                            break;
                        }
                }
                if (pass == 0 && flag == 2) {
                    counter_in++;
                    ED(m, 1, counter_in) = n;
                    ED(m, 2, counter_in) = node;
                    ET(m, 1, counter_in) = elems[0];
                    ET(m, 2, counter_in) = elems[1];
                }
                if (pass == 1 && flag == 1) {
                    counter_in++;
                    ED(m, 1, counter_in) = n;
                    ED(m, 2, counter_in) = node;
                    ET(m, 1, counter_in) = elems[0];
                    ET(m, 2, counter_in) = -999;
                }
            }
        }
        if (pass == 0) m->Ed_in = counter_in;
    }
    /* (d) the first element lies to the left of the edge vector */
    for (int n = 1; n <= m->Ed; ++n) {
        int e1 = ED(m, 1, n), e2 = ED(m, 2, n);
        double xc1, xc2, amin;
        elem_center(m, ET(m, 1, n), &xc1, &xc2, &amin);
        xc1 = xc1 - CX(m, e1);
        xc2 = xc2 - CY(m, e1);
        double xe1 = CX(m, e2) - CX(m, e1), xe2 = CY(m, e2) - CY(m, e1);
        xe1 = cyc_fix(m, xe1);
        xc1 = cyc_fix(m, xc1);
        if (xc1 * xe2 - xc2 * xe1 > 0.0) {
            int el = ET(m, 1, n), el1 = ET(m, 2, n);
            if (el1 > 0) {
                ET(m, 1, n) = el1;
                ET(m, 2, n) = el;
            } else {
                int t = ED(m, 2, n);
                ED(m, 2, n) = ED(m, 1, n);
                ED(m, 1, n) = t;
            }
        }
    }
    /* (e) edges of each element, in the rotation sense of its nodes */
    m->elem_edges = calloc(4 * (size_t)E, sizeof(int32_t));
    int *cnt = calloc((size_t)E + 1, sizeof(int));
    for (int n = 1; n <= m->Ed; ++n)
        for (int k = 1; k <= 2; ++k) {
            int q = ET(m, k, n);
            if (q > 0) {
                cnt[q]++;
                EE(m, cnt[q], q) = n;
            }
        }
    for (int elem = 1; elem <= E; ++elem) {
        int el[4] = {EN(m, 1, elem), EN(m, 2, elem), EN(m, 3, elem), EN(m, 4, elem)};
        int q1 = (el[0] == el[3]) ? 3 : 4;
        int eledges[4] = {EE(m, 1, elem), EE(m, 2, elem), EE(m, 3, elem), EE(m, 4, elem)};
        for (int q = 1; q <= q1 - 1; ++q)
            for (int k = 0; k < q1; ++k) {
                int a = ED(m, 1, eledges[k]), b = ED(m, 2, eledges[k]);
                if ((a == el[q - 1] && b == el[q]) || (a == el[q] && b == el[q - 1])) {
                    EE(m, q, elem) = eledges[k];
                    break;
                }
            }
        for (int k = 0; k < q1; ++k) {
            int a = ED(m, 1, eledges[k]), b = ED(m, 2, eledges[k]);
            if ((a == el[q1 - 1] && b == el[0]) || (a == el[0] && b == el[q1 - 1])) {
                EE(m, q1, elem) = eledges[k];
                break;
            }
        }
        if (q1 == 3) EE(m, 4, elem) = EE(m, 1, elem);
    }
    free(cnt);
    free(ne_num);
    free(ne_pos);
    free(aux1);
    free(nn_num);
    free(nn_pos);
    return FESOMC_OK;
}

/* find_elem_neighbors (fv_mesh_array.F90:791-946), serial build */
static void find_elem_neighbors(oracle_mesh *m) {
    const int E = m->E, N = m->N;
    m->elem_nb = calloc(4 * (size_t)E, sizeof(int32_t));
    for (int elem = 1; elem <= E; ++elem) {
        int e1 = EE(m, 1, elem), e4 = EE(m, 4, elem);
        int q = (e1 == e4 || e4 == 0) ? 3 : 4;
        for (int j = 1; j <= q; ++j) {
            int ed = EE(m, j, elem);
            int el1 = ET(m, 1, ed);
            if (el1 == elem) el1 = ET(m, 2, ed);
            m->elem_nb[4 * (elem - 1) + j - 1] = el1;
        }
        if (q == 3) m->elem_nb[4 * (elem - 1) + 3] = m->elem_nb[4 * (elem - 1)];
    }
    m->nie_num = calloc((size_t)N, sizeof(int32_t));
    for (int el = 1; el <= E; ++el) {
        int q = (EN(m, 1, el) == EN(m, 4, el)) ? 3 : 4;
        for (int j = 1; j <= q; ++j) m->nie_num[EN(m, j, el) - 1]++;
    }
    int mx = 0;
    for (int n = 0; n < N; ++n)
        if (m->nie_num[n] > mx) mx = m->nie_num[n];
    m->nie_max = mx;
    m->nie = calloc((size_t)mx * (size_t)N, sizeof(int32_t));
    memset(m->nie_num, 0, sizeof(int32_t) * (size_t)N);
    for (int el = 1; el <= E; ++el) {
        int q = (EN(m, 1, el) == EN(m, 4, el)) ? 3 : 4;
        for (int j = 1; j <= q; ++j) {
            int nd = EN(m, j, el);
            m->nie_num[nd - 1]++;
            m->nie[(size_t)mx * (nd - 1) + m->nie_num[nd - 1] - 1] = el;
        }
    }
}

/* cdiff (fv_mesh_array.F90:1141-1152): x2 - x1 with the cyclic fix */
static void cdiff(const oracle_mesh *m, const double x2[2], const double x1[2], double xd[2]) {
    double d0 = x2[0] - x1[0], d1 = x2[1] - x1[1];
    d0 = cyc_fix(m, d0);
    xd[0] = d0;
    xd[1] = d1;
}

/* mesh_arrays1 (fv_mesh_array.F90:948-1139) */
static void mesh_arrays1(oracle_mesh *m, int coriolis_on, double lat_deg) {
    const int E = m->E, N = m->N;
    const double omega = 2.0 * O_PI / (3600.0 * 24.0);      /* fv_var.F90:15 */
    m->elem_area = calloc((size_t)E, sizeof(double));
    m->elem_cos = calloc((size_t)E, sizeof(double));
    m->coriolis = calloc((size_t)E, sizeof(double));
    m->area = calloc((size_t)N, sizeof(double));
    m->w_cv = calloc(4 * (size_t)E, sizeof(double));
    for (int elem = 1; elem <= E; ++elem) {
        double ax, ay, aa;
        elem_center(m, elem, &ax, &ay, &aa);
        m->coriolis[elem - 1] = 2.0 * omega * sin(ay);
        m->elem_cos[elem - 1] = cos(ay);
        m->elem_area[elem - 1] = aa;
    }
    if (m->cart)
        for (int e = 0; e < E; ++e) m->elem_cos[e] = 1.0;
    if (coriolis_on) {
        if (m->cart) {
            const double lat_cartesian = lat_deg * O_PI / 180.0;   /* fv_read_run.F90:501 */
            for (int e = 0; e < E; ++e) m->coriolis[e] = 2.0 * omega * sin(lat_cartesian);
        }
    } else {
        for (int e = 0; e < E; ++e) m->coriolis[e] = 0.0;
    }
    for (int e = 0; e < E; ++e) m->elem_area[e] = m->elem_area[e] * m->elem_cos[e];
    for (int elem = 1; elem <= E; ++elem) {
        int eln[6];
        for (int q = 0; q < 4; ++q) eln[q + 1] = EN(m, q + 1, elem);
        double *w = &m->w_cv[4 * (elem - 1)];
        if (eln[1] == eln[4]) {
            for (int j = 2; j <= 4; ++j) {
                m->area[eln[j - 1] - 1] = m->area[eln[j - 1] - 1] + m->elem_area[elem - 1] / 3.0;
                w[j - 2] = 1.0 / 3.0;
            }
        } else {
            double rc[2], aa;
            elem_center(m, elem, &rc[0], &rc[1], &aa);
            eln[0] = eln[4];
            eln[5] = eln[1];
            for (int j = 2; j <= 5; ++j) {
                double r1[2] = {CX(m, eln[j - 2]), CY(m, eln[j - 2])};
                double r0[2] = {CX(m, eln[j - 1]), CY(m, eln[j - 1])};
                double rr[2], rl[2], t[2];
                cdiff(m, r1, r0, rr);
                r1[0] = CX(m, eln[j]);
                r1[1] = CY(m, eln[j]);
                cdiff(m, r1, r0, rl);
                cdiff(m, rc, r0, t);
                r0[0] = t[0];
                r0[1] = t[1];
                const double ec = m->elem_cos[elem - 1];
                const double part = 0.25 * ec * (fabs(rl[0] * r0[1] - rl[1] * r0[0]) + fabs(rr[0] * r0[1] - rr[1] * r0[0]));
                m->area[eln[j - 1] - 1] = m->area[eln[j - 1] - 1] + part;
                w[j - 2] = 0.25 * ec * (fabs(rl[0] * r0[1] - rl[1] * r0[0]) + fabs(rr[0] * r0[1] - rr[1] * r0[0])) /
                           m->elem_area[elem - 1];
            }
        }
    }
    for (int e = 0; e < E; ++e) m->elem_area[e] = m->elem_area[e] * O_REARTH * O_REARTH;
    for (int n = 0; n < N; ++n) m->area[n] = m->area[n] * O_REARTH * O_REARTH;
}

/* mesh_arrays2 (fv_mesh_array.F90:1155-1386) */
static void mesh_arrays2(oracle_mesh *m) {
    const int E = m->E, Ed = m->Ed;
    m->cx = malloc(sizeof(double) * (size_t)E);
    m->cy = malloc(sizeof(double) * (size_t)E);
    m->edxdy = malloc(sizeof(double) * 2 * (size_t)Ed);
    m->ecross = malloc(sizeof(double) * 4 * (size_t)Ed);
    m->gs = calloc(8 * (size_t)E, sizeof(double));
    m->gv = calloc(8 * (size_t)E, sizeof(double));
    for (int n = 1; n <= E; ++n) {
        double aa;
        elem_center(m, n, &m->cx[n - 1], &m->cy[n - 1], &aa);
    }
    for (int n = 1; n <= Ed; ++n) {
        double a0 = CX(m, ED(m, 2, n)) - CX(m, ED(m, 1, n));
        double a1 = CY(m, ED(m, 2, n)) - CY(m, ED(m, 1, n));
        a0 = cyc_fix(m, a0);
        m->edxdy[2 * (n - 1)] = a0;
        m->edxdy[2 * (n - 1) + 1] = a1;
    }
    for (int edg = 1; edg <= Ed; ++edg) {
        int el1 = ET(m, 1, edg), el2 = ET(m, 2, edg);
        double a0, a1;
        edge_center(m, ED(m, 1, edg), ED(m, 2, edg), &a0, &a1);
        double b0 = m->cx[el1 - 1] - a0, b1 = m->cy[el1 - 1] - a1;
        b0 = cyc_fix(m, b0);
        b0 = b0 * m->elem_cos[el1 - 1];
        b0 = b0 * O_REARTH;
        b1 = b1 * O_REARTH;
        double *c = &m->ecross[4 * (edg - 1)];
        c[0] = b0;
        c[1] = b1;
        if (el2 > 0) {
            b0 = m->cx[el2 - 1] - a0;
            b1 = m->cy[el2 - 1] - a1;
            b0 = cyc_fix(m, b0);
            b0 = b0 * m->elem_cos[el2 - 1];
            b0 = b0 * O_REARTH;
            b1 = b1 * O_REARTH;
            c[2] = b0;
            c[3] = b1;
        } else {
            c[2] = 0.0;
            c[3] = 0.0;
        }
    }
    /* derivatives of scalar quantities */
    for (int elem = 1; elem <= E; ++elem) {
        double *g = &m->gs[8 * (elem - 1)];
        const double ec = m->elem_cos[elem - 1];
        if (EN(m, 1, elem) == EN(m, 4, elem)) {
            int n1 = EN(m, 1, elem), n2 = EN(m, 2, elem), n3 = EN(m, 3, elem);
            double dX31 = CX(m, n3) - CX(m, n1);
            dX31 = cyc_fix(m, dX31);
            dX31 = ec * dX31;
            double dX21 = CX(m, n2) - CX(m, n1);
            dX21 = cyc_fix(m, dX21);
            dX21 = ec * dX21;
            double dY31 = CY(m, n3) - CY(m, n1);
            double dY21 = CY(m, n2) - CY(m, n1);
            double dfactor = -0.5 * O_REARTH / m->elem_area[elem - 1];
            g[0] = (-dY31 + dY21) * dfactor;
            g[1] = dY31 * dfactor;
            g[2] = -dY21 * dfactor;
            g[3] = 0.0;
            g[4] = (dX31 - dX21) * dfactor;
            g[5] = -dX31 * dfactor;
            g[6] = dX21 * dfactor;
            g[7] = 0.0;
        } else {
            int en6[6];
            for (int q = 0; q < 4; ++q) en6[q + 1] = EN(m, q + 1, elem);
            en6[0] = en6[4];
            en6[5] = en6[1];
            double dfactor = 0.5 * O_REARTH / m->elem_area[elem - 1];
            for (int j = 2; j <= 5; ++j) {
                double x1[2] = {CX(m, en6[j - 1]), CY(m, en6[j - 1])};
                double x2[2] = {CX(m, en6[j - 2]), CY(m, en6[j - 2])};
                double xd[2], x3[2];
                cdiff(m, x1, x2, xd);
                x2[0] = CX(m, en6[j]);
                x2[1] = CY(m, en6[j]);
                cdiff(m, x2, x1, x3);
                xd[0] = xd[0] + x3[0];
                xd[1] = xd[1] + x3[1];
                xd[0] = xd[0] * ec;
                g[j - 2] = -xd[1] * dfactor;
                g[j - 2 + 4] = xd[0] * dfactor;
            }
        }
    }
    /* derivatives of vector quantities: least squares over the neighbours */
    for (int elem = 1; elem <= E; ++elem) {
        double a0 = m->cx[elem - 1], a1 = m->cy[elem - 1];
        int q = (EN(m, 1, elem) == EN(m, 4, elem)) ? 3 : 4;
        double x[4], y[4];
        for (int j = 1; j <= q; ++j) {
            int el = m->elem_nb[4 * (elem - 1) + j - 1];
            if (el > 0) {
                x[j - 1] = m->cx[el - 1] - a0;
                x[j - 1] = cyc_fix(m, x[j - 1]);
                y[j - 1] = m->cy[el - 1] - a1;
            } else {
                int ed = EE(m, j, elem);
                double b0, b1;
                edge_center(m, ED(m, 1, ed), ED(m, 2, ed), &b0, &b1);
                x[j - 1] = (b0 - a0);
                x[j - 1] = cyc_fix(m, x[j - 1]);
                x[j - 1] = 2.0 * x[j - 1];
                y[j - 1] = 2.0 * (b1 - a1);
            }
        }
        if (q == 3) {
            x[3] = 0.0;
            y[3] = 0.0;
        }
        const double ec = m->elem_cos[elem - 1];
        for (int j = 0; j < 4; ++j) {
            x[j] = x[j] * ec * O_REARTH;
            y[j] = y[j] * O_REARTH;
        }
        double cxx = x[0] * x[0], cxy = x[0] * y[0], cyy = y[0] * y[0];
        for (int j = 1; j < 4; ++j) {
            cxx = cxx + x[j] * x[j];
            cxy = cxy + x[j] * y[j];
            cyy = cyy + y[j] * y[j];
        }
        double d = cxy * cxy - cxx * cyy;
        double *g = &m->gv[8 * (elem - 1)];
        for (int j = 0; j < 4; ++j) {
            g[j] = (cxy * y[j] - cyy * x[j]) / d;
            g[j + 4] = (cxy * x[j] - cxx * y[j]) / d;
        }
    }
}

/* the two element sides b, c at node nd of element elem, as
 * find_up_downwind_triangles takes them (fv_mesh_array.F90:1486-1510) */
static void sides_at(const oracle_mesh *m, int elem, int nd, double b[2], double c[2]) {
#define P(k, i) (i == 0 ? CX(m, EN(m, k, elem)) : CY(m, EN(m, k, elem)))
    int tri = EN(m, 1, elem) == EN(m, 4, elem);
    int o, pb, pc;                                /* origin, b end, c end */
    if (tri) {
        if (EN(m, 1, elem) == nd) { o = 1; pb = 2; pc = 3; }
        else if (EN(m, 2, elem) == nd) { o = 2; pb = 1; pc = 3; }
        else { o = 3; pb = 1; pc = 2; }
    } else {
        if (EN(m, 1, elem) == nd) { o = 1; pb = 2; pc = 4; }
        else if (EN(m, 2, elem) == nd) { o = 2; pb = 3; pc = 1; }
        else if (EN(m, 3, elem) == nd) { o = 3; pb = 4; pc = 2; }
        else { o = 4; pb = 1; pc = 3; }
    }
    for (int i = 0; i < 2; ++i) {
        b[i] = P(pb, i) - P(o, i);
        c[i] = P(pc, i) - P(o, i);
    }
#undef P
    b[0] = cyc_fix(m, b[0]);
    c[0] = cyc_fix(m, c[0]);
}

/* does vector x lie between the sides b and c (the three accepting tests) */
static int between(const double b[2], const double c[2], const double x[2]) {
    double cr = c[0] * c[0] + c[1] * c[1];
    double bx = (b[0] * c[0] + b[1] * c[1]) / cr;
    double by = (-b[0] * c[1] + b[1] * c[0]) / cr;
    double xx = (x[0] * c[0] + x[1] * c[1]) / cr;
    double xy = (-x[0] * c[1] + x[1] * c[0]) / cr;
    double ab = atan2(by, bx);
    double ax = atan2(xy, xx);
    if ((ab > 0) && (ax > 0) && (ax < ab)) return 1;
    if ((ab < 0) && (ax < 0) && (ax > ab)) return 1;
    if ((ab == ax) || (ax == 0.0)) return 1;
    return 0;
}

/* find_up_downwind_triangles (fv_mesh_array.F90:1390-1618): the element at
 * each end of an edge that contains the edge direction continued backwards
 * (up) or forwards (down); when several do, the last one in nod_in_elem2D
 * order (the Fortran loop goes on after each hit) */
static void find_up_dn(oracle_mesh *m) {
    m->updn = calloc(2 * (size_t)m->Ed, sizeof(int32_t));
    for (int n = 1; n <= m->Ed; ++n) {
        int n1 = ED(m, 1, n), n2 = ED(m, 2, n);
        double x[2] = {CX(m, n2) - CX(m, n1), CY(m, n2) - CY(m, n1)};
        x[0] = cyc_fix(m, x[0]);
        x[0] = -x[0];
        x[1] = -x[1];
        for (int k = 0; k < m->nie_num[n1 - 1]; ++k) {
            int elem = m->nie[(size_t)m->nie_max * (n1 - 1) + k];
            double b[2], c[2];
            sides_at(m, elem, n1, b, c);
            if (between(b, c, x)) m->updn[2 * (n - 1)] = elem;
        }
        x[0] = -x[0];
        x[1] = -x[1];
        for (int k = 0; k < m->nie_num[n2 - 1]; ++k) {
            int elem = m->nie[(size_t)m->nie_max * (n2 - 1) + k];
            double b[2], c[2];
            sides_at(m, elem, n2, b, c);
            if (between(b, c, x)) m->updn[2 * (n - 1) + 1] = elem;
        }
    }
}

/* SET_SIGMA, cases 1 and 2 (fv_vert_coord.F90:135-200) */
static int set_sigma(oracle_mesh *m, const fesomc_mesh_opts *o) {
    const int ns = o->nsigma;
    m->sigma = malloc(sizeof(double) * (size_t)ns);
    if (o->ind_sigma == 1) {
        if (o->pow_sig > 1 && ns % 2 == 0) return FESOMC_EINVAL;
        if (o->pow_sig == 1) {
            for (int K = 1; K <= ns; ++K) m->sigma[K - 1] = -pow((K - 1) / (double)(ns - 1), o->pow_sig) + 1.0;
        } else {
            for (int K = 1; K <= (ns + 1) / 2; ++K)
                m->sigma[K - 1] = -pow((K - 1) / (double)((ns + 1) / 2 - 1), o->pow_sig) * 0.5 + 1.0;
            for (int K = (ns + 1) / 2 + 1; K <= ns; ++K)
                m->sigma[K - 1] = pow((ns - K) / (double)((ns + 1) / 2 - 1), o->pow_sig) * 0.5;
        }
    } else if (o->ind_sigma == 2) {
        for (int K = 1; K <= ns; ++K) {
            double X1 = tanh((o->lev_bot + o->lev_sur) * (ns - K) / (ns - 1) - o->lev_bot);
            double X2 = tanh(o->lev_bot);
            double X3 = X2 + tanh(o->lev_sur);
            m->sigma[K - 1] = (X1 + X2) / X3;
        }
    } else {
        return FESOMC_EINVAL;
    }
    return FESOMC_OK;
}

void oracle_mesh_free(oracle_mesh *m) {
    if (!m) return;
    void *ps[] = {m->index, m->en, m->edge_nodes, m->edge_tri, m->elem_edges, m->elem_nb, m->nie_num, m->nie,
                  m->updn, m->in_obn, m->rivers, m->coord, m->depth, m->area, m->elem_area, m->elem_cos,
                  m->coriolis, m->w_cv, m->gs, m->gv, m->edxdy, m->ecross, m->sigma, m->a_tp, m->ac, m->cx, m->cy};
    for (size_t i = 0; i < sizeof(ps) / sizeof(ps[0]); ++i) free(ps[i]);
    free(m);
}

/* Same inputs and outputs as fesomc_mesh_build: node coordinates as in
 * nod2d.out (metres if cartesian, degrees otherwise), node flags, elements as
 * in elem2d.out (4 per row, node4 = node1 for triangles, 1-based), depth. */
int oracle_mesh_build(int32_t nod2D, const double *xy, const int32_t *index_nod2D, int32_t elem2D,
                      const int32_t *elem_nodes4, const double *depth, const fesomc_mesh_opts *o,
                      oracle_mesh **out) {
    if (!xy || !index_nod2D || !elem_nodes4 || !depth || !o || !out || nod2D < 3 || elem2D < 1) return FESOMC_EINVAL;
    *out = NULL;
    oracle_mesh *m = calloc(1, sizeof(oracle_mesh));
    if (!m) return FESOMC_ENOMEM;
    m->N = nod2D;
    m->E = elem2D;
    m->NS = o->nsigma;
    m->cart = o->cartesian != 0;
    m->cyc = o->cyclic_length_deg * O_RAD;                 /* fv_read_run.F90:622 */
    /* read_mesh_ser: coordinates, open-boundary list, triangles first */
    m->coord = malloc(sizeof(double) * 2 * (size_t)nod2D);
    m->index = malloc(sizeof(int32_t) * (size_t)nod2D);
    m->depth = malloc(sizeof(double) * (size_t)nod2D);
    for (int n = 0; n < nod2D; ++n) {
        m->index[n] = index_nod2D[n];
        m->depth[n] = depth[n];
        if (m->cart) {
            m->coord[2 * n] = xy[2 * n] / O_REARTH;
            m->coord[2 * n + 1] = xy[2 * n + 1] / O_REARTH;
        } else {
            m->coord[2 * n] = xy[2 * n] * O_RAD;
            m->coord[2 * n + 1] = xy[2 * n + 1] * O_RAD;
        }
        if (index_nod2D[n] == 2) m->nobn++;
    }
    m->in_obn = malloc(sizeof(int32_t) * (size_t)(m->nobn > 0 ? m->nobn : 1));
    for (int n = 0, k = 0; n < nod2D; ++n)
        if (index_nod2D[n] == 2) m->in_obn[k++] = n + 1;
    m->en = malloc(sizeof(int32_t) * 4 * (size_t)elem2D);
    int ntri = 0;
    for (int pass = 0; pass < 2; ++pass)
        for (int e = 0; e < elem2D; ++e) {
            const int32_t *nd = &elem_nodes4[4 * e];
            if ((pass == 0) == (nd[0] == nd[3])) {
                for (int q = 0; q < 4; ++q) {
                    if (nd[q] < 1 || nd[q] > nod2D) {
                        oracle_mesh_free(m);
                        return FESOMC_EINVAL;
                    }
                    m->en[4 * ntri + q] = nd[q];
                }
                ntri++;
            }
        }
    int rc = test_elem(m);
    if (!rc) rc = find_edges(m);
    if (rc) {
        oracle_mesh_free(m);
        return rc;
    }
    find_elem_neighbors(m);
    mesh_arrays1(m, o->coriolis_on, o->lat_cartesian_deg);
    mesh_arrays2(m);
    if (o->with_up_dn_tri) find_up_dn(m);
    if ((rc = set_sigma(m, o))) {
        oracle_mesh_free(m);
        return rc;
    }
    /* a_tp (fv_ini.F90:94-107), stored (nod2D, 2) */
    m->a_tp = malloc(sizeof(double) * 2 * (size_t)nod2D);
    for (int n = 0; n < nod2D; ++n) {
        m->a_tp[n] = o->T_potential ? 0.918 : 1.0;
        m->a_tp[nod2D + n] = o->T_potential ? 0.69 : 0.0;
        if (m->index[n] == 2) {
            m->a_tp[n] = 1.0;
            m->a_tp[nod2D + n] = 0.0;
        }
    }
    m->ac = malloc(sizeof(double) * (size_t)nod2D);
    for (int n = 0; n < nod2D; ++n) m->ac[n] = 1.0;
    *out = m;
    return FESOMC_OK;
}

int oracle_mesh_view(const oracle_mesh *m, fesomc_mesh *v) {
    if (!m || !v) return FESOMC_EINVAL;
    memset(v, 0, sizeof(*v));
    v->nod2D = m->N;
    v->elem2D = m->E;
    v->edge2D = m->Ed;
    v->edge2D_in = m->Ed_in;
    v->nsigma = m->NS;
    v->nod_in_elem2D_max = m->nie_max;
    v->index_nod2D = m->index;
    v->elem2D_nodes = m->en;
    v->edge_nodes = m->edge_nodes;
    v->edge_tri = m->edge_tri;
    v->elem_edges = m->elem_edges;
    v->elem_neighbors = m->elem_nb;
    v->nod_in_elem2D_num = m->nie_num;
    v->nod_in_elem2D = m->nie;
    v->edge_up_dn_tri = m->updn;
    v->coord_nod2D = m->coord;
    v->depth = m->depth;
    v->area = m->area;
    v->elem_area = m->elem_area;
    v->elem_cos = m->elem_cos;
    v->coriolis = m->coriolis;
    v->w_cv = m->w_cv;
    v->gradient_sca = m->gs;
    v->gradient_vec = m->gv;
    v->edge_dxdy = m->edxdy;
    v->edge_cross_dxdy = m->ecross;
    v->sigma = m->sigma;
    v->a_tp = m->a_tp;
    v->ac = m->ac;
    v->nobn = m->nobn;
    v->in_obn = m->in_obn;
    v->n_rivers = m->nriv;
    v->nod_rivers = m->rivers;
    return FESOMC_OK;
}

/* scale_area = sum(elem_area)/elem2D, sequential sum (fv_ini.F90:81) */
double oracle_mesh_scale_area(const oracle_mesh *m) {
    double s = 0.0;
    for (int e = 0; e < m->E; ++e) s = s + m->elem_area[e];
    return s / m->E;
}

int oracle_mesh_set_rivers(oracle_mesh *m, int32_t n, const int32_t *nodes) {
    if (!m || n < 0 || (n > 0 && !nodes)) return FESOMC_EINVAL;
    free(m->rivers);
    m->rivers = malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) {
        if (nodes[i] < 1 || nodes[i] > m->N) return FESOMC_EINVAL;
        m->rivers[i] = nodes[i];
    }
    m->nriv = n;
    return FESOMC_OK;
}

/* ac_create with Dist2in1 (fv_utilit.F90:53-88,184-220): ac = d/radius
 * inside the sponge, 1 elsewhere, d the distance to the nearest open-boundary
 * node (Euclidean on the scaled cartesian coordinates, haversine otherwise;
 * Fortran precedence makes cos_X2 * cos(X2obn) * sin(..)**2 the product
 * (cos_X2 * cos) * (s * s)) */
int oracle_mesh_set_sponge(oracle_mesh *m, double radius) {
    if (!m || !(radius > 0.0)) return FESOMC_EINVAL;
    for (int n = 0; n < m->N; ++n) m->ac[n] = 1.0;
    if (m->nobn == 0) return FESOMC_OK;
    for (int n = 0; n < m->N; ++n) {
        const double X1 = m->coord[2 * n], X2 = m->coord[2 * n + 1];
        double d2obn;
        if (m->cart) {
            double d = 0.0;
            for (int j = 0; j < m->nobn; ++j) {
                const int k = m->in_obn[j] - 1;
                const double dx = m->coord[2 * k] - X1, dy = m->coord[2 * k + 1] - X2;
                const double v = dx * dx + dy * dy;
                if (j == 0 || v < d) d = v;
            }
            d2obn = sqrt(d) * O_REARTH;
        } else {
            const double cos_X2 = cos(X2);
            double a = 0.0;
            for (int j = 0; j < m->nobn; ++j) {
                const int k = m->in_obn[j] - 1;
                const double s1 = sin((m->coord[2 * k + 1] - X2) * 0.5);
                const double s2 = sin((m->coord[2 * k] - X1) * 0.5);
                const double v = s1 * s1 + cos_X2 * cos(m->coord[2 * k + 1]) * (s2 * s2);
                if (j == 0 || v < a) a = v;
            }
            d2obn = 2.0 * O_REARTH * asin(fmin(1.0, sqrt(a)));
        }
        if (d2obn < radius) m->ac[n] = d2obn / radius;
    }
    return FESOMC_OK;
}
