/*
 * mph_oracle.c — CPU restatement of the MPH-WC explicit time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
 * compared against; it is never linked into the product library and the
 * product never calls it.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load it.
 *
 * It restates, in plain C with the dimension as a run-time value, the
 * algorithm of Masahiro-Kondo-AIST/MphExplicit source/main.cpp.  Each function
 * cites the lines it follows.  Floating-point expressions keep the reference's
 * operation order so that, compiled without FMA contraction
 * (-ffp-contract=off, no -ffast-math), it reproduces the reference bit for
 * bit.  Pinned against the reference compiled from its own sources
 * (oracle/_ref, built by oracle/Makefile) and against committed fixtures
 * (tests/golden/).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include "mph_b200.h"

#define TC MPH_TYPE_COUNT
#define IS_FLUID(t) ((t) >= 0 && (t) < 2)   /* FLUID_BEGIN..FLUID_END, main.cpp:44-45 */
#define IS_WALL(t)  ((t) >= 2 && (t) < 4)   /* WALL_BEGIN..WALL_END,   main.cpp:46-47 */

typedef struct oracle_state {
    int dim, n;
    mph_params p;
    mph_grid_header h;
    mph_constants c;
    double time;
    long long steps, rebuilds;
    double wall_center[TC][3];
    /* per particle, current (cell-sorted) order */
    int *pidx, *type, *ncount;
    double (*x)[3], (*v)[3], (*f)[3], (*snap)[3];
    double *mass, *kappa, *lambda_, *mu;
    double *dens_a, (*gc)[3], *pres_a, *strain_p, *div_p, *pres_p;
    double *vir_p, (*vir_s)[3][3];
    /* cells */
    int pow2, pow2_exp, *cell_index, *cell_particle;
    int *cfb, *cfe, *cwb, *cwe;
    int fluid_begin, fluid_end, wall_begin, wall_end;
    long long *nptr;
    int *nind;
    long long nind_count;
    int *tmp_i;
    double (*tmp_v)[3];
} oracle_state;

/* Mod macro, main.cpp:70 */
static inline double omod(double x, double w) { return x - w * floor(x / w); }

/* Kernel shapes, main.cpp:214-284.  hp() is h*h in 2-D and h*h*h in 3-D. */
static inline double hp(const oracle_state* s, double h) { return s->dim == 2 ? h * h : h * h * h; }
static double k_wa(const oracle_state* s, double r, double h) {
    return 1.0 / s->c.swa * 1.0 / hp(s, h) * (r / h) * (1.0 - (r / h)) * (1.0 - (r / h));
}
static double k_dwadr(const oracle_state* s, double r, double h) {
    return 1.0 / s->c.swa * 1.0 / hp(s, h) * (1.0 - (r / h)) * (1.0 - 3.0 * (r / h)) * (1.0 / h);
}
static double k_wg(const oracle_state* s, double r, double h) {
    return 1.0 / s->c.swg * 1.0 / hp(s, h) * ((1.0 - r / h) * (1.0 - r / h));
}
static double k_dwgdr(const oracle_state* s, double r, double h) {
    return 1.0 / s->c.swg * 1.0 / hp(s, h) * (-2.0 / h * (1.0 - r / h));
}
static double k_wp(const oracle_state* s, double r, double h) {
    return 1.0 / s->c.swp * 1.0 / hp(s, h) * ((1.0 - r / h) * (1.0 - r / h));
}
static double k_dwpdr(const oracle_state* s, double r, double h) {
    return 1.0 / s->c.swp * 1.0 / hp(s, h) * (-2.0 / h * (1.0 - r / h));
}
static double k_dwvdr(const oracle_state* s, double r, double h) {
    return 1.0 / s->c.swv * 1.0 / hp(s, h) * (-2.0 / h * (1.0 - r / h));
}

/* minimum-image displacement x_j - x_i (main.cpp:1680, identical in every sweep) */
static inline void disp(const oracle_state* s, const double* xi, const double* xj, double* out) {
    for (int d = 0; d < 3; ++d) {
        const double w = s->c.domain_width[d];
        out[d] = omod(xj[d] - xi[d] + 0.5 * w, w) - 0.5 * w;
    }
}

/* ---------------------------------------------------------------------- */
/* set-up: initializeWeight main.cpp:836-954, initializeFluid 971-983,
 * initializeWall 994-1033, initializeDomain 1035-1084 */
int oracle_compute_constants(const mph_params* p, const mph_grid_header* h, int dim, mph_constants* c) {
    if (!p || !h || !c || (dim != 2 && dim != 3)) return MPH_ERR_ARG;
    memset(c, 0, sizeof(*c));
    const double l0 = h->particle_spacing;
    c->dim = dim;
    c->particle_volume = dim == 2 ? l0 * l0 : l0 * l0 * l0;               /* main.cpp:558-562 */
    const double rrg = p->radius_ratio_a;                                  /* main.cpp:838 */
    c->radius_a = p->radius_ratio_a * l0;
    c->radius_g = rrg * l0;
    c->radius_p = p->radius_ratio_p * l0;
    c->radius_v = p->radius_ratio_v * l0;
    if (dim == 2) {                                                        /* main.cpp:846-851 */
        c->swa = 1.0 / 2.0 * 2.0 / 15.0 * M_PI / l0 / l0;
        c->swg = 1.0 / 2.0 * 1.0 / 3.0 * M_PI / l0 / l0;
        c->swp = 1.0 / 2.0 * 1.0 / 3.0 * M_PI / l0 / l0;
        c->swv = 1.0 / 2.0 * 1.0 / 3.0 * M_PI / l0 / l0;
        c->r2g = 1.0 / 2.0 * 1.0 / 30.0 * M_PI * c->radius_g * c->radius_g / l0 / l0 / c->swg;
    } else {                                                               /* main.cpp:853-857 */
        c->swa = 1.0 / 3.0 * 1.0 / 5.0 * M_PI / l0 / l0 / l0;
        c->swg = 1.0 / 3.0 * 2.0 / 5.0 * M_PI / l0 / l0 / l0;
        c->swp = 1.0 / 3.0 * 2.0 / 5.0 * M_PI / l0 / l0 / l0;
        c->swv = 1.0 / 3.0 * 2.0 / 5.0 * M_PI / l0 / l0 / l0;
        c->r2g = 1.0 / 3.0 * 4.0 / 105.0 * M_PI * c->radius_g * c->radius_g / l0 / l0 / l0 / c->swg;
    }
    /* N0a / N0p lattice sums, main.cpp:861-949: origin excluded, r^2 <= R^2 inclusive */
    oracle_state tmp;
    memset(&tmp, 0, sizeof(tmp));
    tmp.dim = dim;
    tmp.c = *c;
    for (int which = 0; which < 2; ++which) {
        const double radius = which == 0 ? c->radius_a : c->radius_p;
        const int range = (int)(radius / l0 + 3.0);
        const int zr = dim == 2 ? 0 : range;
        int count = 0;
        double sum = 0.0;
        for (int ix = -range; ix <= range; ++ix)
            for (int iy = -range; iy <= range; ++iy)
                for (int iz = -zr; iz <= zr; ++iz) {
                    if (ix == 0 && iy == 0 && iz == 0) continue;
                    const double x = l0 * ((double)ix), y = l0 * ((double)iy), z = l0 * ((double)iz);
                    const double rij2 = dim == 2 ? x * x + y * y : x * x + y * y + z * z;
                    if (rij2 <= radius * radius) {
                        const double rij = sqrt(rij2);
                        sum += which == 0 ? k_wa(&tmp, rij, radius) : k_wp(&tmp, rij, radius);
                        count++;
                    }
                }
        if (which == 0) { c->n0a = sum; c->n0a_count = count; }
        else            { c->n0p = sum; c->n0p_count = count; }
    }
    /* CofK / CofA, main.cpp:971-983 */
    double integN, integX;
    if (dim == 2) { c->cof_k = 0.350778153; integN = 0.024679383; integX = 0.226126699; }
    else          { c->cof_k = 0.326976006; integN = 0.021425779; integX = 0.233977488; }
    for (int t = 0; t < TC; ++t)
        c->cof_a[t] = p->surface_tension[t] / ((c->radius_g / l0) * (integN + c->cof_k * c->cof_k * integX));
    /* wall rotation, main.cpp:997-1031 (theta = |w|^2 without sqrt, as the reference has it) */
    for (int t = 2; t < TC; ++t) {
        double normal[3] = {0.0, 0.0, 0.0}, q[4];
        const double* w = p->wall_omega[t];
        const double theta = fabs(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        if (theta != 0.0)
            for (int d = 0; d < 3; ++d) normal[d] = w[d] / theta;
        q[0] = normal[0] * sin(theta * p->dt / 2.0);
        q[1] = normal[1] * sin(theta * p->dt / 2.0);
        q[2] = normal[2] * sin(theta * p->dt / 2.0);
        q[3] = cos(theta * p->dt / 2.0);
        double (*R)[3] = c->wall_rotation[t];
        R[0][0] = q[0] * q[0] - q[1] * q[1] - q[2] * q[2] + q[3] * q[3];
        R[0][1] = 2.0 * (q[0] * q[1] - q[2] * q[3]);
        R[0][2] = 2.0 * (q[0] * q[2] + q[1] * q[3]);
        R[1][0] = 2.0 * (q[0] * q[1] + q[2] * q[3]);
        R[1][1] = -q[0] * q[0] + q[1] * q[1] - q[2] * q[2] + q[3] * q[3];
        R[1][2] = 2.0 * (q[1] * q[2] - q[0] * q[3]);
        R[2][0] = 2.0 * (q[0] * q[2] - q[1] * q[3]);
        R[2][1] = 2.0 * (q[1] * q[2] + q[0] * q[3]);
        R[2][2] = -q[0] * q[0] - q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    }
    /* initializeDomain, main.cpp:1039-1067 */
    double mr = 0.0;
    mr = c->radius_a > mr ? c->radius_a : mr;
    mr = c->radius_g > mr ? c->radius_g : mr;
    mr = c->radius_p > mr ? c->radius_p : mr;
    mr = c->radius_v > mr ? c->radius_v : mr;
    c->max_radius = mr;
    const double margin = 0.1 * l0;                                         /* MARGIN, main.cpp:89 */
    double cc[3];
    for (int d = 0; d < 3; ++d) c->domain_width[d] = h->domain_max[d] - h->domain_min[d];
    cc[0] = floor((h->domain_max[0] - h->domain_min[0]) / (mr + margin));
    cc[1] = floor((h->domain_max[1] - h->domain_min[1]) / (mr + margin));
    cc[2] = dim == 2 ? 1 : floor((h->domain_max[2] - h->domain_min[2]) / (mr + margin));
    for (int d = 0; d < 3; ++d) c->cell_count[d] = (int)cc[d];
    c->total_cell_count = (int)(cc[0] * cc[1] * cc[2]);
    for (int d = 0; d < 3; ++d) c->cell_width[d] = c->domain_width[d] / c->cell_count[d];
    return MPH_OK;
}

/* ---------------------------------------------------------------------- */
static inline int cell_id(const oracle_state* s, int ix, int iy, int iz) {   /* main.cpp:96-100 */
    const int* C = s->c.cell_count;
    return ((ix % C[0] + C[0]) % C[0]) * C[1] * C[2] + ((iy % C[1] + C[1]) % C[1]) * C[2]
           + ((iz % C[2] + C[2]) % C[2]);
}

/* calculateCellParticle, main.cpp:1111-1326 */
static void cell_particle(oracle_state* s) {
    const int n = s->n, P = s->pow2, tot = s->c.total_cell_count;
    const int* C = s->c.cell_count;
    const double* dmin = s->h.domain_min;
    const double* cw = s->c.cell_width;
    for (int i = 0; i < P; ++i) {                                           /* 1118-1133 */
        if (i < n) {
            const int cx = ((int)floor((s->x[i][0] - dmin[0]) / cw[0])) % C[0];
            const int cy = ((int)floor((s->x[i][1] - dmin[1]) / cw[1])) % C[1];
            const int cz = ((int)floor((s->x[i][2] - dmin[2]) / cw[2])) % C[2];
            s->cell_index[i] = cell_id(s, cx, cy, cz);
            if (IS_WALL(s->type[i])) s->cell_index[i] += tot;
            s->cell_particle[i] = i;
        } else {
            s->cell_index[i] = 2 * tot;
            s->cell_particle[i] = n;
        }
    }
    /* bitonic network, 1137-1158: pass (m, k) compares i and i|2^(m-k) */
    for (int m = 0; m < s->pow2_exp; ++m)
        for (int k = 0; k <= m; ++k) {
            const int dist = 1 << (m - k);
            for (int i = 0; i < P; ++i) {
                const int up = ((i >> m) & 2) == 0;
                if ((i & dist) == 0 && ((s->cell_index[i] > s->cell_index[i | dist]) == up)) {
                    int t = s->cell_index[i]; s->cell_index[i] = s->cell_index[i | dist]; s->cell_index[i | dist] = t;
                    t = s->cell_particle[i]; s->cell_particle[i] = s->cell_particle[i | dist]; s->cell_particle[i | dist] = t;
                }
            }
        }
    /* per-cell ranges, 1160-1247.  The reference detects boundaries and then
     * rebuilds every begin/end from a prefix sum of the per-cell counts, so
     * begin(b) is the number of sorted keys below b for every key value b. */
    {
        int pos = 0;
        for (int b = 0; b <= 2 * tot; ++b) {
            while (pos < n && s->cell_index[pos] < b) ++pos;
            /* pos = #keys < b */
            if (b < tot) s->cfb[b] = pos;
            if (b >= 1 && b <= tot) s->cfe[b - 1] = pos;
            if (b >= tot && b < 2 * tot) s->cwb[b - tot] = pos;
            if (b >= tot + 1) s->cwe[b - tot - 1] = pos;
        }
    }
    s->fluid_begin = s->cfb[0];                                             /* 1252-1258 */
    s->fluid_end = s->cfe[tot - 1];
    s->wall_begin = s->cwb[0];
    s->wall_end = s->cwe[tot - 1];
    /* gather-reorder, 1262-1325 */
    for (int i = 0; i < n; ++i) s->tmp_i[i] = s->pidx[s->cell_particle[i]];
    memcpy(s->pidx, s->tmp_i, sizeof(int) * n);
    for (int i = 0; i < n; ++i) s->tmp_i[i] = s->type[s->cell_particle[i]];
    memcpy(s->type, s->tmp_i, sizeof(int) * n);
    for (int i = 0; i < n; ++i) memcpy(s->tmp_v[i], s->x[s->cell_particle[i]], sizeof(double) * 3);
    memcpy(s->x, s->tmp_v, sizeof(double) * 3 * n);
    for (int i = 0; i < n; ++i) memcpy(s->tmp_v[i], s->v[s->cell_particle[i]], sizeof(double) * 3);
    memcpy(s->v, s->tmp_v, sizeof(double) * 3 * n);
}

/* the 3^D stencil of cell ids in the reference's visiting order, main.cpp:1356-1392 */
static int stencil(const oracle_state* s, int i, int* cells) {
    const int* C = s->c.cell_count;
    const int tot = s->c.total_cell_count;
    const double rm = s->c.max_radius + 0.1 * s->h.particle_spacing;
    const int rx = (int)ceil(rm / s->c.cell_width[0]);
    const int ry = (int)ceil(rm / s->c.cell_width[1]);
    const int rz = s->dim == 2 ? 0 : (int)ceil(rm / s->c.cell_width[2]);
    const int ci = s->cell_index[i];
    const int icx = (ci / (C[1] * C[2])) % tot;
    const int icy = (ci / C[2]) % C[1];
    const int icz = ci % C[2];
    int jcx[3], jcy[3], jcz[3];
    for (int j = 0; j < 2 * rx + 1; ++j) jcx[j] = ((icx - rx + j) % C[0] + C[0]) % C[0];
    for (int j = 0; j < 2 * ry + 1; ++j) jcy[j] = ((icy - ry + j) % C[1] + C[1]) % C[1];
    for (int j = 0; j < 2 * rz + 1; ++j) jcz[j] = ((icz - rz + j) % C[2] + C[2]) % C[2];
    const int bx = (2 * rx) - (icx + rx) % C[0], xmin = bx > 0 ? bx : 0;
    const int by = (2 * ry) - (icy + ry) % C[1], ymin = by > 0 ? by : 0;
    const int bz = (2 * rz) - (icz + rz) % C[2], zmin = bz > 0 ? bz : 0;
    int k = 0;
    for (int jx = xmin; jx < xmin + (2 * rx + 1); ++jx)
        for (int jy = ymin; jy < ymin + (2 * ry + 1); ++jy)
            for (int jz = zmin; jz < zmin + (2 * rz + 1); ++jz)
                cells[k++] = cell_id(s, jcx[jx % (2 * rx + 1)], jcy[jy % (2 * ry + 1)], jcz[jz % (2 * rz + 1)]);
    return k;
}

/* calculateNeighbor, main.cpp:1329-1596 (count pass, scan, fill pass, snapshot) */
static int neighbor(oracle_state* s) {
    const int n = s->n;
    const double rm = s->c.max_radius + 0.1 * s->h.particle_spacing;
    const double rm2 = rm * rm;
    {   /* asserts of main.cpp:1347-1349 */
        const int rx = (int)ceil(rm / s->c.cell_width[0]);
        const int ry = (int)ceil(rm / s->c.cell_width[1]);
        const int rz = s->dim == 2 ? 0 : (int)ceil(rm / s->c.cell_width[2]);
        if (2 * rx + 1 > 3 || 2 * ry + 1 > 3 || 2 * rz + 1 > 3) return MPH_ERR_GEOMETRY;
    }
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {                                                   /* 1452-1494 */
            s->nptr[0] = 0;
            for (int i = 0; i < n; ++i) s->nptr[i + 1] = s->nptr[i] + s->ncount[i];
            s->nind_count = s->nptr[n];
            free(s->nind);
            s->nind = (int*)malloc(sizeof(int) * (size_t)(s->nind_count > 0 ? s->nind_count : 1));
        }
#pragma omp parallel for schedule(dynamic, 256)
        for (int i = 0; i < n; ++i) {
            int cells[27];
            const int nc = stencil(s, i, cells);
            int cnt = 0;
            int* out = pass ? s->nind + s->nptr[i] : NULL;
            for (int kind = 0; kind < 2; ++kind) {
                /* 1416 / 1557: a wall particle with no fluid neighbour skips the wall cells */
                if (kind == 1 && s->wall_begin <= i && i < s->wall_end && cnt == 0) break;
                for (int k = 0; k < nc; ++k) {
                    const int cc = cells[k];
                    const int b = kind == 0 ? s->cfb[cc] : s->cwb[cc];
                    const int e = kind == 0 ? s->cfe[cc] : s->cwe[cc];
                    for (int j = b; j < e; ++j) {
                        double q[3];
                        disp(s, s->x[i], s->x[j], q);
                        const double q2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
                        if (q2 <= rm2) {
                            if (out) out[cnt] = j;
                            cnt++;
                        }
                    }
                }
            }
            if (!pass) s->ncount[i] = cnt;
        }
    }
    memcpy(s->snap, s->x, sizeof(double) * 3 * n);                          /* 1587-1595 */
    return MPH_OK;
}

/* neighborCalculation, main.cpp:1086-1108 */
static int need_rebuild(const oracle_state* s) {
    double mx = 0.0;
    for (int i = 0; i < s->n; ++i) {
        double d[3];
        for (int k = 0; k < 3; ++k) {
            const double w = s->c.domain_width[k];
            d[k] = omod(s->x[i][k] - s->snap[i][k] + 0.5 * w, w) - 0.5 * w;
        }
        const double sh = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        if (sh > mx) mx = sh;
    }
    const double margin = 0.1 * s->h.particle_spacing;
    return mx > 0.5 * margin * 0.5 * margin;
}

#define NLOOP(i) for (int jn = 0; jn < s->ncount[i]; ++jn)
#define NJ(i) (s->nind[s->nptr[i] + jn])

/* calculateDensityA, main.cpp:1665-1692 */
static void density_a(oracle_state* s) {
    const double R = s->c.radius_a;
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < s->n; ++i) {
        double sum = 0.0;
        NLOOP(i) {
            const int j = NJ(i);
            if (i == j) continue;
            const double ratio = s->p.interaction_ratio[s->type[i]][s->type[j]];
            double x[3];
            disp(s, s->x[i], s->x[j], x);
            const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            if (R * R - r2 >= 0) sum += ratio * k_wa(s, sqrt(r2), R);
        }
        s->dens_a[i] = sum;
    }
}

/* calculateGravityCenter, main.cpp:1695-1727 */
static void gravity_center(oracle_state* s) {
    const double R = s->c.radius_g;
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < s->n; ++i) {
        double sum[3] = {0.0, 0.0, 0.0};
        NLOOP(i) {
            const int j = NJ(i);
            if (i == j) continue;
            const double ratio = s->p.interaction_ratio[s->type[i]][s->type[j]];
            double x[3];
            disp(s, s->x[i], s->x[j], x);
            const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            if (R * R - r2 >= 0) {
                const double w = ratio * k_wg(s, sqrt(r2), R);
                for (int d = 0; d < 3; ++d) sum[d] += x[d] * w / s->c.r2g * R;
            }
        }
        for (int d = 0; d < 3; ++d) s->gc[i][d] = sum[d];
    }
}

/* calculateDensityP, main.cpp:1831-1858 */
static void density_p(oracle_state* s) {
    const double R = s->c.radius_p;
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < s->n; ++i) {
        double sum = 0.0;
        NLOOP(i) {
            const int j = NJ(i);
            if (i == j) continue;
            double x[3];
            disp(s, s->x[i], s->x[j], x);
            const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            if (R * R - r2 >= 0) sum += k_wp(s, sqrt(r2), R);
        }
        s->strain_p[i] = sum - s->c.n0p;
    }
}

/* calculateDivergenceP, main.cpp:1860-1896 */
static void divergence_p(oracle_state* s) {
    const double R = s->c.radius_p;
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < s->n; ++i) {
        double sum = 0.0;
        NLOOP(i) {
            const int j = NJ(i);
            if (i == j) continue;
            double x[3];
            disp(s, s->x[i], s->x[j], x);
            const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            if (R * R - r2 >= 0) {
                const double r = sqrt(r2);
                const double dw = k_dwpdr(s, r, R);
                const double e[3] = {x[0] / r, x[1] / r, x[2] / r};
                double u[3];
                for (int d = 0; d < 3; ++d) u[d] = s->v[j][d] - s->v[i][d];
                for (int d = 0; d < 3; ++d) sum -= u[d] * e[d] * dw;
            }
        }
        s->div_p[i] = sum;
    }
}

/* calculatePhysicalCoefficients, main.cpp:1631-1662 */
static void physical_coefficients(oracle_state* s) {
    for (int i = 0; i < s->n; ++i) {
        const int t = s->type[i];
        s->mass[i] = s->p.density[t] * s->c.particle_volume;
        s->kappa[i] = s->p.bulk_modulus[t];
        if (s->strain_p[i] < 0.0) s->kappa[i] = 0.0;
        s->lambda_[i] = s->p.bulk_viscosity[t];
        s->mu[i] = s->p.shear_viscosity[t];
    }
}

/* calculatePressureP, main.cpp:1898-1939 */
static void pressure_p(oracle_state* s) {
    const double R = s->c.radius_p, V = s->c.particle_volume;
    for (int i = 0; i < s->n; ++i) s->pres_p[i] = -s->lambda_[i] * s->div_p[i] + s->kappa[i] * s->strain_p[i];
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < s->n; ++i) {
        double f[3] = {0.0, 0.0, 0.0};
        NLOOP(i) {
            const int j = NJ(i);
            if (i == j) continue;
            double x[3];
            disp(s, s->x[i], s->x[j], x);
            const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            if (R * R - r2 > 0) {
                const double r = sqrt(r2);
                const double dw = k_dwpdr(s, r, R);
                const double g[3] = {dw * x[0] / r, dw * x[1] / r, dw * x[2] / r};
                for (int d = 0; d < 3; ++d) f[d] += (s->pres_p[i] + s->pres_p[j]) * g[d] * V;
            }
        }
        for (int d = 0; d < 3; ++d) s->f[i][d] += f[d];
    }
}

/* calculatePressureA, main.cpp:1729-1776 */
static void pressure_a(oracle_state* s) {
    const double R = s->c.radius_a, V = s->c.particle_volume, l0 = s->h.particle_spacing;
    for (int i = 0; i < s->n; ++i) {
        s->pres_a[i] = s->c.cof_a[s->type[i]] * (s->dens_a[i] - s->c.n0a) / l0;
        if (s->c.n0a <= s->dens_a[i]) s->pres_a[i] = 0.0;
    }
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < s->n; ++i) {
        double f[3] = {0.0, 0.0, 0.0};
        NLOOP(i) {
            const int j = NJ(i);
            if (i == j) continue;
            const double rij_ = s->p.interaction_ratio[s->type[i]][s->type[j]];
            const double rji_ = s->p.interaction_ratio[s->type[j]][s->type[i]];
            double x[3];
            disp(s, s->x[i], s->x[j], x);
            const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            if (R * R - r2 > 0) {
                const double r = sqrt(r2);
                const double dwij = rij_ * k_dwadr(s, r, R);
                const double dwji = rji_ * k_dwadr(s, r, R);
                const double e[3] = {x[0] / r, x[1] / r, x[2] / r};
                for (int d = 0; d < 3; ++d) f[d] += (s->pres_a[i] * dwij + s->pres_a[j] * dwji) * e[d] * V;
            }
        }
        for (int d = 0; d < 3; ++d) s->f[i][d] += f[d];
    }
}

/* calculateDiffuseInterface, main.cpp:1778-1829 (aj uses the type of i, as in the reference) */
static void diffuse_interface(oracle_state* s) {
    const double R = s->c.radius_g, V = s->c.particle_volume, l0 = s->h.particle_spacing;
    const double ck = s->c.cof_k, r2g = s->c.r2g;
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < s->n; ++i) {
        const double ai = s->c.cof_a[s->type[i]] * (ck) * (ck);
        double f[3] = {0.0, 0.0, 0.0};
        NLOOP(i) {
            const int j = NJ(i);
            if (i == j) continue;
            const double aj = s->c.cof_a[s->type[i]] * (ck) * (ck);
            const double rij_ = s->p.interaction_ratio[s->type[i]][s->type[j]];
            const double rji_ = s->p.interaction_ratio[s->type[j]][s->type[i]];
            double x[3];
            disp(s, s->x[i], s->x[j], x);
            const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            if (R * R - r2 > 0) {
                const double r = sqrt(r2);
                const double wij = rij_ * k_wg(s, r, R);
                const double wji = rji_ * k_wg(s, r, R);
                for (int d = 0; d < 3; ++d)
                    f[d] -= (aj * s->gc[j][d] * wji - ai * s->gc[i][d] * wij) / r2g * R * (V / l0);
                const double dwij = rij_ * k_dwgdr(s, r, R);
                const double dwji = rji_ * k_dwgdr(s, r, R);
                const double e[3] = {x[0] / r, x[1] / r, x[2] / r};
                double gr = 0.0;
                for (int d = 0; d < 3; ++d) gr += (aj * s->gc[j][d] * dwji - ai * s->gc[i][d] * dwij) * x[d];
                for (int d = 0; d < 3; ++d) f[d] -= (gr) * e[d] / r2g * R * (V / l0);
            }
        }
        for (int d = 0; d < 3; ++d) s->f[i][d] += f[d];
    }
}

/* calculateViscosityV, main.cpp:1941-1985 */
static void viscosity_v(oracle_state* s) {
    const double R = s->c.radius_v, V = s->c.particle_volume;
    const double cv = s->dim == 2 ? 8.0 : 10.0;
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < s->n; ++i) {
        double f[3] = {0.0, 0.0, 0.0};
        NLOOP(i) {
            const int j = NJ(i);
            if (i == j) continue;
            double x[3];
            disp(s, s->x[i], s->x[j], x);
            const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
            if (R * R - r2 > 0) {
                const double r = sqrt(r2);
                const double dw = -k_dwvdr(s, r, R);
                const double e[3] = {x[0] / r, x[1] / r, x[2] / r};
                double u[3];
                for (int d = 0; d < 3; ++d) u[d] = s->v[j][d] - s->v[i][d];
                const double muij = 2.0 * (s->mu[i] * s->mu[j]) / (s->mu[i] + s->mu[j]);
                for (int d = 0; d < 3; ++d)
                    f[d] += cv * muij * (u[0] * e[0] + u[1] * e[1] + u[2] * e[2]) * e[d] * dw / r * V;
            }
        }
        for (int d = 0; d < 3; ++d) s->f[i][d] += f[d];
    }
}

/* calculateVirialStressAtParticle, main.cpp:2057-2302 */
static void virial(oracle_state* s) {
    const double V = s->c.particle_volume, l0 = s->h.particle_spacing;
    const double cv = s->dim == 2 ? 8.0 : 10.0;
    memset(s->vir_s, 0, sizeof(double) * 9 * s->n);
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < s->n; ++i) {
        for (int term = 0; term < 4; ++term) {
            double st[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            NLOOP(i) {
                const int j = NJ(i);
                if (i == j) continue;
                double x[3];
                disp(s, s->x[i], s->x[j], x);
                const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
                double fij[3];
                if (term == 0) {                                           /* 2092-2109 */
                    const double R = s->c.radius_p;
                    if (!(R * R - r2 > 0)) continue;
                    const double r = sqrt(r2);
                    const double dw = k_dwpdr(s, r, R);
                    const double g[3] = {dw * x[0] / r, dw * x[1] / r, dw * x[2] / r};
                    for (int d = 0; d < 3; ++d) fij[d] = (s->pres_p[i]) * g[d] * V;
                    for (int a = 0; a < 3; ++a)
                        for (int b = 0; b < 3; ++b) st[a][b] += 1.0 * fij[a] * x[b] / V;
                } else if (term == 1) {                                    /* 2137-2155 */
                    const double R = s->c.radius_a;
                    if (!(R * R - r2 > 0)) continue;
                    const double ratio = s->p.interaction_ratio[s->type[i]][s->type[j]];
                    const double r = sqrt(r2);
                    const double dw = ratio * k_dwadr(s, r, R);
                    const double g[3] = {dw * x[0] / r, dw * x[1] / r, dw * x[2] / r};
                    for (int d = 0; d < 3; ++d) fij[d] = (s->pres_a[i]) * g[d] * V;
                    for (int a = 0; a < 3; ++a)
                        for (int b = 0; b < 3; ++b) st[a][b] += 1.0 * fij[a] * x[b] / V;
                } else if (term == 2) {                                    /* 2184-2207 */
                    const double R = s->c.radius_v;
                    if (!(R * R - r2 > 0)) continue;
                    const double r = sqrt(r2);
                    const double dw = -k_dwvdr(s, r, R);
                    const double e[3] = {x[0] / r, x[1] / r, x[2] / r};
                    const double u[3] = {s->v[j][0] - s->v[i][0], s->v[j][1] - s->v[i][1], s->v[j][2] - s->v[i][2]};
                    const double muij = 2.0 * (s->mu[i] * s->mu[j]) / (s->mu[i] + s->mu[j]);
                    for (int d = 0; d < 3; ++d)
                        fij[d] = cv * muij * (u[0] * e[0] + u[1] * e[1] + u[2] * e[2]) * e[d] * dw / r * V;
                    for (int a = 0; a < 3; ++a)
                        for (int b = 0; b < 3; ++b) st[a][b] += 0.5 * fij[a] * x[b] / V;
                } else {                                                   /* 2235-2279 */
                    const double R = s->c.radius_g;
                    if (R * R - r2 > 0) {
                        const double a = s->c.cof_a[s->type[i]] * (s->c.cof_k) * (s->c.cof_k);
                        const double ratio = s->p.interaction_ratio[s->type[i]][s->type[j]];
                        const double r = sqrt(r2);
                        const double w = ratio * k_wg(s, r, R);
                        for (int d = 0; d < 3; ++d)
                            fij[d] = -a * (-s->gc[i][d]) * w / s->c.r2g * R * (V / l0);
                        for (int aa = 0; aa < 3; ++aa)
                            for (int b = 0; b < 3; ++b) st[aa][b] += 1.0 * fij[aa] * x[b] / V;
                    }
                    if (R * R - r2 > 0.0) {
                        const double a = s->c.cof_a[s->type[i]] * (s->c.cof_k) * (s->c.cof_k);
                        const double ratio = s->p.interaction_ratio[s->type[i]][s->type[j]];
                        const double r = sqrt(r2);
                        const double dw = ratio * k_dwgdr(s, r, R);
                        const double g[3] = {dw * x[0] / r, dw * x[1] / r, dw * x[2] / r};
                        double gr = 0.0;
                        for (int d = 0; d < 3; ++d) gr += (-s->gc[i][d]) * x[d];
                        for (int d = 0; d < 3; ++d)
                            fij[d] = -a * (gr) * g[d] / s->c.r2g * R * (V / l0);
                        for (int aa = 0; aa < 3; ++aa)
                            for (int b = 0; b < 3; ++b) st[aa][b] += 1.0 * fij[aa] * x[b] / V;
                    }
                }
            }
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) s->vir_s[i][a][b] += st[a][b];
        }
        if (s->dim == 2) s->vir_p[i] = -1.0 / 2.0 * (s->vir_s[i][0][0] + s->vir_s[i][1][1]);
        else s->vir_p[i] = -1.0 / 3.0 * (s->vir_s[i][0][0] + s->vir_s[i][1][1] + s->vir_s[i][2][2]);
    }
}

/* calculateConvection 1605-1615, calculateWall 2013-2053, calculatePeriodicBoundary 2306-2317,
 * resetForce 1617-1628 */
static void move(oracle_state* s) {
    const double dt = s->p.dt;
    for (int i = s->fluid_begin; i < s->fluid_end; ++i)
        for (int d = 0; d < 3; ++d) s->x[i][d] += s->v[i][d] * dt;
    for (int i = s->wall_begin; i < s->wall_end; ++i) {
        const int t = s->type[i];
        const double* C = s->wall_center[t];
        const double* W = s->p.wall_omega[t];
        const double* U = s->p.wall_velocity[t];
        const double (*R)[3] = (const double (*)[3])s->c.wall_rotation[t];
        s->f[i][0] = s->f[i][1] = s->f[i][2] = 0.0;
        double r[3] = {s->x[i][0] - C[0], s->x[i][1] - C[1], s->x[i][2] - C[2]};
        r[0] = R[0][0] * r[0] + R[0][1] * r[1] + R[0][2] * r[2];
        r[1] = R[1][0] * r[0] + R[1][1] * r[1] + R[1][2] * r[2];
        r[2] = R[2][0] * r[0] + R[2][1] * r[1] + R[2][2] * r[2];
        s->v[i][0] = W[1] * r[2] - W[2] * r[1] + U[0];
        s->v[i][1] = W[2] * r[0] - W[0] * r[2] + U[1];
        s->v[i][2] = W[0] * r[1] - W[1] * r[0] + U[2];
        s->x[i][0] = r[0] + C[0] + U[0] * dt;
        s->x[i][1] = r[1] + C[1] + U[1] * dt;
        s->x[i][2] = r[2] + C[2] + U[2] * dt;
    }
    for (int t = 2; t < TC; ++t)
        for (int d = 0; d < 3; ++d) s->wall_center[t][d] += s->p.wall_velocity[t][d] * dt;
    for (int i = 0; i < s->n; ++i)
        for (int d = 0; d < 3; ++d)
            s->x[i][d] = omod(s->x[i][d] - s->h.domain_min[d], s->c.domain_width[d]) + s->h.domain_min[d];
    memset(s->f, 0, sizeof(double) * 3 * s->n);
}

/* calculateGravity 1988-1998, calculateAcceleration 2000-2010 */
static void accelerate(oracle_state* s) {
    for (int i = s->fluid_begin; i < s->fluid_end; ++i)
        for (int d = 0; d < 3; ++d) s->f[i][d] += s->mass[i] * s->p.gravity[d];
    for (int i = s->fluid_begin; i < s->fluid_end; ++i)
        for (int d = 0; d < 3; ++d) s->v[i][d] += s->f[i][d] / s->mass[i] * s->p.dt;
}

/* ---------------------------------------------------------------------- */
/* public (test-only) interface */

void oracle_destroy(oracle_state* s) {
    if (!s) return;
    void* ptrs[] = {s->pidx, s->type, s->ncount, s->x, s->v, s->f, s->snap, s->mass, s->kappa,
                    s->lambda_, s->mu, s->dens_a, s->gc, s->pres_a, s->strain_p, s->div_p,
                    s->pres_p, s->vir_p, s->vir_s, s->cell_index, s->cell_particle, s->cfb,
                    s->cfe, s->cwb, s->cwe, s->nptr, s->nind, s->tmp_i, s->tmp_v};
    for (size_t k = 0; k < sizeof(ptrs) / sizeof(ptrs[0]); ++k) free(ptrs[k]);
    free(s);
}

/* set-up and start-up sequence of main(), main.cpp:324-364 */
oracle_state* oracle_create(const mph_params* p, const mph_grid_header* h, int dim,
                            const int* type, const double* xyz, const double* vel) {
    if (!p || !h || !type || !xyz || !vel || h->particle_count <= 0) return NULL;
    oracle_state* s = (oracle_state*)calloc(1, sizeof(oracle_state));
    s->dim = dim;
    s->n = h->particle_count;
    s->p = *p;
    s->h = *h;
    s->time = h->time;
    if (oracle_compute_constants(p, h, dim, &s->c) != MPH_OK) { free(s); return NULL; }
    memcpy(s->wall_center, p->wall_center, sizeof(s->wall_center));
    const int n = s->n;
    s->pidx = (int*)malloc(sizeof(int) * n);
    s->type = (int*)malloc(sizeof(int) * n);
    s->ncount = (int*)calloc(n, sizeof(int));
    s->x = (double (*)[3])malloc(sizeof(double) * 3 * n);
    s->v = (double (*)[3])malloc(sizeof(double) * 3 * n);
    s->f = (double (*)[3])calloc(3 * (size_t)n, sizeof(double));
    s->snap = (double (*)[3])malloc(sizeof(double) * 3 * n);
    s->mass = (double*)malloc(sizeof(double) * n);
    s->kappa = (double*)malloc(sizeof(double) * n);
    s->lambda_ = (double*)malloc(sizeof(double) * n);
    s->mu = (double*)malloc(sizeof(double) * n);
    s->dens_a = (double*)calloc(n, sizeof(double));
    s->gc = (double (*)[3])calloc(3 * (size_t)n, sizeof(double));
    s->pres_a = (double*)calloc(n, sizeof(double));
    s->strain_p = (double*)calloc(n, sizeof(double));
    s->div_p = (double*)calloc(n, sizeof(double));
    s->pres_p = (double*)calloc(n, sizeof(double));
    s->vir_p = (double*)calloc(n, sizeof(double));
    s->vir_s = (double (*)[3][3])calloc(9 * (size_t)n, sizeof(double));
    s->tmp_i = (int*)malloc(sizeof(int) * n);
    s->tmp_v = (double (*)[3])malloc(sizeof(double) * 3 * n);
    /* main.cpp:612-617: smallest power of two strictly above n */
    s->pow2_exp = 0;
    while ((n >> s->pow2_exp) != 0) ++s->pow2_exp;
    s->pow2 = 1 << s->pow2_exp;
    s->cell_index = (int*)malloc(sizeof(int) * s->pow2);
    s->cell_particle = (int*)malloc(sizeof(int) * s->pow2);
    const int tot = s->c.total_cell_count;
    s->cfb = (int*)malloc(sizeof(int) * tot);
    s->cfe = (int*)malloc(sizeof(int) * tot);
    s->cwb = (int*)malloc(sizeof(int) * tot);
    s->cwe = (int*)malloc(sizeof(int) * tot);
    s->nptr = (long long*)calloc((size_t)n + 1, sizeof(long long));
    s->nind = NULL;
    memcpy(s->type, type, sizeof(int) * n);
    memcpy(s->x, xyz, sizeof(double) * 3 * n);
    memcpy(s->v, vel, sizeof(double) * 3 * n);
    for (int i = 0; i < n; ++i) {
        s->pidx[i] = i;                                                    /* main.cpp:645-647 */
        if (type[i] < 0 || type[i] >= TC) { oracle_destroy(s); return NULL; }
    }
    for (int i = 0; i < n; ++i) {                                          /* initializeFluid 959-970 */
        s->mass[i] = p->density[type[i]] * s->c.particle_volume;
        s->kappa[i] = p->bulk_modulus[type[i]];
        s->lambda_[i] = p->bulk_viscosity[type[i]];
        s->mu[i] = p->shear_viscosity[type[i]];
    }
    cell_particle(s);                                                      /* main.cpp:358-364 */
    if (neighbor(s) != MPH_OK) { oracle_destroy(s); return NULL; }
    density_a(s);
    gravity_center(s);
    density_p(s);
    return s;
}

/* the loop body main.cpp:386-431 and Time += Dt (449) */
void oracle_step(oracle_state* s, int nsteps) {
    for (int k = 0; k < nsteps; ++k) {
        move(s);
        if (need_rebuild(s)) {
            cell_particle(s);
            neighbor(s);
            s->rebuilds++;
        }
        density_a(s);
        gravity_center(s);
        density_p(s);
        divergence_p(s);
        physical_coefficients(s);
        pressure_p(s);
        pressure_a(s);
        diffuse_interface(s);
        viscosity_v(s);
        accelerate(s);
        s->time += s->p.dt;
        s->steps++;
    }
}

void oracle_virial(oracle_state* s) { virial(s); }

int oracle_particle_count(const oracle_state* s) { return s->n; }
long long oracle_rebuild_count(const oracle_state* s) { return s->rebuilds; }
long long oracle_neighbor_ind_count(const oracle_state* s) { return s->nind_count; }
double oracle_time(const oracle_state* s) { return s->time; }
void oracle_get_constants(const oracle_state* s, mph_constants* c) { *c = s->c; }

void oracle_get_state(const oracle_state* s, int* pidx, int* type, double* xyz, double* vel,
                      double* force, int* ncount, double* dens_a, double* strain_p, double* vir_p) {
    const size_t n = (size_t)s->n;
    if (pidx) memcpy(pidx, s->pidx, sizeof(int) * n);
    if (type) memcpy(type, s->type, sizeof(int) * n);
    if (xyz) memcpy(xyz, s->x, sizeof(double) * 3 * n);
    if (vel) memcpy(vel, s->v, sizeof(double) * 3 * n);
    if (force) memcpy(force, s->f, sizeof(double) * 3 * n);
    if (ncount) memcpy(ncount, s->ncount, sizeof(int) * n);
    if (dens_a) memcpy(dens_a, s->dens_a, sizeof(double) * n);
    if (strain_p) memcpy(strain_p, s->strain_p, sizeof(double) * n);
    if (vir_p) memcpy(vir_p, s->vir_p, sizeof(double) * n);
}

void oracle_get_fields(const oracle_state* s, double* div_p, double* pres_p, double* pres_a, double* gc) {
    const size_t n = (size_t)s->n;
    if (div_p) memcpy(div_p, s->div_p, sizeof(double) * n);
    if (pres_p) memcpy(pres_p, s->pres_p, sizeof(double) * n);
    if (pres_a) memcpy(pres_a, s->pres_a, sizeof(double) * n);
    if (gc) memcpy(gc, s->gc, sizeof(double) * 3 * n);
}

void oracle_get_cells(const oracle_state* s, int* cell_index, int* fb, int* fe, int* wb, int* we) {
    const int tot = s->c.total_cell_count;
    if (cell_index) memcpy(cell_index, s->cell_index, sizeof(int) * s->n);
    if (fb) memcpy(fb, s->cfb, sizeof(int) * tot);
    if (fe) memcpy(fe, s->cfe, sizeof(int) * tot);
    if (wb) memcpy(wb, s->cwb, sizeof(int) * tot);
    if (we) memcpy(we, s->cwe, sizeof(int) * tot);
}

void oracle_get_neighbors(const oracle_state* s, long long* ptr, int* ind) {
    if (ptr) memcpy(ptr, s->nptr, sizeof(long long) * ((size_t)s->n + 1));
    if (ind) memcpy(ind, s->nind, sizeof(int) * (size_t)s->nind_count);
}
