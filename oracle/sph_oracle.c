/*
 * Test infrastructure only: CPU oracle for the emerald 2D SPH step.
 *
 * A plain-C restatement of the reference algorithm, function by function:
 *   emerald/z_index/z_index.{h,cpp}            Morton keys
 *   emerald/sph_common/ (.h, .cpp)             grid, sort, neighbours, kernels,
 *                                              density, divergence, pressure,
 *                                              dynamics, CFL, reductions
 *   emerald/sph2d_box/ (.h, .cpp)              IISPH, IISPH_AP, IISPH_PSEUDO_AP,
 *                                              DFSPH_P and PCISPH sub-steps and
 *                                              the adaptive frame loop
 * Tests check this restatement against the reference compiled from its own
 * sources (oracle/_ref) and then use it to check the CUDA path. The product
 * never links or calls it. Parity: pinned bit-for-bit against oracle/_ref on
 * the scenes exercised by tests/test_oracle_vs_reference.py.
 *
 * Arithmetic: IEEE single precision in the reference's operator order; the
 * file must be compiled with -ffp-contract=off. Per-particle loops are
 * independent (owner writes) and the convergence reductions are integer sums
 * and float maxima, so the OpenMP thread count does not change any bit.
 */
#include "sph_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define NMAX ORACLE_MAX_NEIGHBORS
#define FLICKS_PER_SECOND 705600000.0

typedef struct {
    float x, y;
} v2;

static inline v2 mk(float x, float y) {
    v2 r;
    r.x = x;
    r.y = y;
    return r;
}
static inline v2 add(v2 a, v2 b) { return mk(a.x + b.x, a.y + b.y); }
static inline v2 sub(v2 a, v2 b) { return mk(a.x - b.x, a.y - b.y); }
static inline v2 neg(v2 a) { return mk(-a.x, -a.y); }
static inline v2 scl(float s, v2 a) { return mk(s * a.x, s * a.y); }
static inline v2 divs(v2 a, float s) { return mk(a.x / s, a.y / s); }
static inline float dot(v2 a, v2 b) { return a.x * b.x + a.y * b.y; }
static inline float sqrf(float a) { return a * a; }
/* std::max(0.0f, x) and std::max(x, 0.0f) differ for NaN and -0.0. */
static inline float max_0x(float x) { return (0.0f < x) ? x : 0.0f; }
static inline float max_x0(float x) { return (x < 0.0f) ? 0.0f : x; }

/* Imath Vec2<float>::length (OpenEXR 2.x): sqrt of the dot product, with the
 * rescaled evaluation for dot < 2*FLT_MIN. */
static float length(v2 a) {
    float const l2 = dot(a, a);
    if (l2 < 2.0f * FLT_MIN) {
        float ax = (a.x >= 0.0f) ? a.x : -a.x;
        float ay = (a.y >= 0.0f) ? a.y : -a.y;
        float m = ax;
        if (m < ay) m = ay;
        if (m == 0.0f) return 0.0f;
        ax /= m;
        ay /= m;
        return m * sqrtf(ax * ax + ay * ay);
    }
    return sqrtf(l2);
}

/* emerald/util/safe_divide.h:20-31 (scalar) and :48-59 (Vec2). */
static inline int safe_f(float n, float d) {
    if (d == 0.0f) return 0;
    if (fabsf(d) >= 1.0f) return 1;
    return (fabsf(d) / FLT_MIN) > fabsf(n);
}
static inline int safe_v(v2 n, float d) {
    if (d == 0.0f) return 0;
    if (fabsf(d) >= 1.0f) return 1;
    float const mr = fabsf(d) / FLT_MIN;
    return (mr > fabsf(n.x)) && (mr > fabsf(n.y));
}
static inline int safe_d(double n, double d) {
    if (d == 0.0) return 0;
    if (fabs(d) >= 1.0) return 1;
    return (fabs(d) / DBL_MIN) > fabs(n);
}

/* emerald/util/functions.h:45-49 */
static inline float mix(float a, float b, float t) { return (a * (1.0f - t)) + (b * t); }

/* ---------------------------------------------------------------- z_index */

/* Single_axis_index<2,BIT>: bit b of i moves to bit 2b
 * (emerald/z_index/z_index.h:11-24); the reference applies it through a
 * 16-bit look-up table to each half of the 32-bit coordinate
 * (emerald/z_index/z_index.cpp:17-44). */
static uint64_t spread16(uint32_t v) {
    uint64_t r = 0;
    for (int b = 0; b < 16; ++b) r |= ((uint64_t)((v >> b) & 1u)) << (2 * b);
    return r;
}
static uint64_t spread32(uint32_t v) {
    return spread16(v & 0xffffu) | (spread16(v >> 16) << 32);
}
/* emerald/z_index/z_index.cpp:8-10, :46-48 */
uint64_t oracle_z_index(uint32_t x, uint32_t y) { return spread32(x) | (spread32(y) << 1); }

/* ---------------------------------------------------------------- kernels */

static float const PI_F = 3.14159274101257324218750f; /* kernels.h:12 */

/* emerald/sph_common/kernels.h:16-23 */
static inline float wa(float q) { return 1.0f + q * q * (q * 0.75f - 1.5f); }
static inline float wb(float q_in) {
    float const q = 2.0f - q_in;
    return (q * q * q) / 4.0f;
}
/* emerald/sph_common/kernels.h:25-35 */
static inline float kw(float r, float h) {
    float const q = r / h;
    float const k = h * h * h * PI_F;
    if (q <= 1.0f) return wa(q) / k;
    if (q <= 2.0f) return wb(q) / k;
    return 0.0f;
}
/* emerald/sph_common/kernels.h:37-55 */
static inline float kdw(float r, float h) {
    float const q = r / h;
    float const k = h * h * h * PI_F;
    if (q <= 1.0f) return (-3.0f * r / (h * h) + 2.25f * r * r / (h * h * h)) / k;
    if (q <= 2.0f) return (-3.0f * sqrf(2.0f - (r / h)) / (4.0f * h)) / k;
    return 0.0f;
}
/* emerald/sph_common/kernels.h:57-64 */
static inline v2 kgradw(v2 dp, float h) {
    float const r = length(dp);
    if (safe_v(dp, r)) {
        float const d = kdw(r, h);
        v2 const u = divs(dp, r);
        return mk(u.x * d, u.y * d);
    }
    return mk(0.0f, 0.0f);
}

float oracle_kernel_w(float r, float h) { return kw(r, h); }
void oracle_kernel_grad_w(float dx, float dy, float h, float* out) {
    v2 const g = kgradw(mk(dx, dy), h);
    out[0] = g.x;
    out[1] = g.y;
}
float oracle_vec2_length(float x, float y) { return length(mk(x, y)); }

/* ------------------------------------------------------ grid, sort, cells */

typedef struct {
    uint64_t z;
    uint64_t i;
} zpair;

static int zpair_cmp(void const* pa, void const* pb) {
    zpair const* a = (zpair const*)pa;
    zpair const* b = (zpair const*)pb;
    if (a->z != b->z) return a->z < b->z ? -1 : 1;
    if (a->i != b->i) return a->i < b->i ? -1 : 1;
    return 0;
}

/* emerald/sph_common/common.cpp:43-56 with bounds_min = (0,0)
 * (emerald/sph2d_box/neighborhoods_from_state.cpp:15-19). */
static inline void grid_coord(v2 p, float cell, int32_t* gx, int32_t* gy) {
    v2 const q = divs(sub(p, mk(0.0f, 0.0f)), cell);
    *gx = (int32_t)floorf(q.x);
    *gy = (int32_t)floorf(q.y);
}

/* The sorted (z, index) pairs and their cell ranges: the outputs of
 * compute_index_pairs / sort_index_pairs / compute_block_indices / fill_blocks
 * (emerald/sph_common/neighborhood.cpp:10-106). Cell lookup by binary search
 * over the unique keys replaces the reference's hash map
 * (create_block_map, :108-124) with the same z -> [begin, end) mapping. */
typedef struct {
    size_t n;
    zpair* pairs;
    size_t ncells;
    uint64_t* cell_z;
    size_t* cell_begin;
    size_t* cell_end;
} cell_index;

static void cell_index_build(cell_index* ci, v2 const* x, size_t n, float cell) {
    ci->n = n;
    ci->pairs = (zpair*)malloc((n ? n : 1) * sizeof(zpair));
    for (size_t i = 0; i < n; ++i) {
        int32_t gx, gy;
        grid_coord(x[i], cell, &gx, &gy);
        ci->pairs[i].z = oracle_z_index((uint32_t)gx, (uint32_t)gy);
        ci->pairs[i].i = i;
    }
    qsort(ci->pairs, n, sizeof(zpair), zpair_cmp);
    ci->cell_z = (uint64_t*)malloc((n ? n : 1) * sizeof(uint64_t));
    ci->cell_begin = (size_t*)malloc((n ? n : 1) * sizeof(size_t));
    ci->cell_end = (size_t*)malloc((n ? n : 1) * sizeof(size_t));
    ci->ncells = 0;
    for (size_t s = 0; s < n; ++s) {
        if (s == 0 || ci->pairs[s].z != ci->pairs[s - 1].z) {
            if (ci->ncells) ci->cell_end[ci->ncells - 1] = s;
            ci->cell_z[ci->ncells] = ci->pairs[s].z;
            ci->cell_begin[ci->ncells] = s;
            ++ci->ncells;
        }
    }
    if (ci->ncells) ci->cell_end[ci->ncells - 1] = n;
}

static void cell_index_free(cell_index* ci) {
    free(ci->pairs);
    free(ci->cell_z);
    free(ci->cell_begin);
    free(ci->cell_end);
    memset(ci, 0, sizeof(*ci));
}

static int cell_lookup(cell_index const* ci, uint64_t z, size_t* b, size_t* e) {
    size_t lo = 0, hi = ci->ncells;
    while (lo < hi) {
        size_t const mid = lo + (hi - lo) / 2;
        if (ci->cell_z[mid] < z) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    if (lo < ci->ncells && ci->cell_z[lo] == z) {
        *b = ci->cell_begin[lo];
        *e = ci->cell_end[lo];
        return 1;
    }
    return 0;
}

size_t oracle_sort(float const* xy,
                   size_t n,
                   float cell_size,
                   int32_t* grid_coords,
                   uint64_t* z_indices,
                   uint64_t* pair_z,
                   uint64_t* pair_index,
                   uint32_t* block_indices,
                   uint64_t* blocks) {
    v2 const* x = (v2 const*)xy;
    cell_index ci;
    cell_index_build(&ci, x, n, cell_size);
    uint32_t block = 0;
    for (size_t i = 0; i < n; ++i) {
        int32_t gx, gy;
        grid_coord(x[i], cell_size, &gx, &gy);
        if (grid_coords) {
            grid_coords[2 * i] = gx;
            grid_coords[2 * i + 1] = gy;
        }
        if (z_indices) z_indices[i] = oracle_z_index((uint32_t)gx, (uint32_t)gy);
        if (pair_z) pair_z[i] = ci.pairs[i].z;
        if (pair_index) pair_index[i] = ci.pairs[i].i;
        if (i > 0 && ci.pairs[i].z != ci.pairs[i - 1].z) ++block;
        if (block_indices) block_indices[i] = block;
    }
    if (blocks) {
        for (size_t c = 0; c < ci.ncells; ++c) {
            blocks[2 * c] = ci.cell_begin[c];
            blocks[2 * c + 1] = ci.cell_end[c];
        }
    }
    size_t const nc = ci.ncells;
    cell_index_free(&ci);
    return nc;
}

/* ------------------------------------------------------------ neighbours */

typedef struct {
    size_t n;
    uint8_t* counts;
    uint32_t* idx; /* n x 64 */
    float* dist;   /* n x 64 */
    v2* vec;       /* n x 64 */
    float* w;      /* n x 64 */
    v2* gw;        /* n x 64 */
} nbhd;

static void nbhd_alloc(nbhd* nb, size_t n) {
    size_t const m = (n ? n : 1) * NMAX;
    nb->n = n;
    nb->counts = (uint8_t*)calloc(n ? n : 1, 1);
    nb->idx = (uint32_t*)calloc(m, sizeof(uint32_t));
    nb->dist = (float*)calloc(m, sizeof(float));
    nb->vec = (v2*)calloc(m, sizeof(v2));
    nb->w = (float*)calloc(m, sizeof(float));
    nb->gw = (v2*)calloc(m, sizeof(v2));
}

static void nbhd_free(nbhd* nb) {
    free(nb->counts);
    free(nb->idx);
    free(nb->dist);
    free(nb->vec);
    free(nb->w);
    free(nb->gw);
    memset(nb, 0, sizeof(*nb));
}

typedef struct {
    uint32_t index;
    float distance;
    v2 vector_to;
} nbr;

/* neighbor_order, emerald/sph_common/neighborhood.h:172-180 */
static int nbr_less(nbr const* a, nbr const* b) {
    if (a->distance < b->distance) return 1;
    if (a->distance > b->distance) return 0;
    return a->index < b->index;
}

/* create_neighborhoods, emerald/sph_common/neighborhood.h:199-282: 3x3 cells
 * in row-major order around the particle's own cell, members in sorted
 * (z, index) order, self skipped for a same-set build, distance < max
 * accepted, at most 64 kept, then ordered by (distance, index). */
static void build_one(size_t i,
                      v2 const* self,
                      v2 const* other,
                      int same_set,
                      cell_index const* ci,
                      float cell,
                      float max_distance,
                      nbhd* out) {
    v2 const pos = self[i];
    int32_t gx, gy;
    grid_coord(pos, cell, &gx, &gy);
    nbr list[NMAX];
    int cnt = 0;
    for (int32_t j = gy - 1; cnt < NMAX && j <= gy + 1; ++j) {
        for (int32_t k = gx - 1; cnt < NMAX && k <= gx + 1; ++k) {
            size_t b, e;
            if (!cell_lookup(ci, oracle_z_index((uint32_t)k, (uint32_t)j), &b, &e)) continue;
            for (size_t s = b; cnt < NMAX && s != e; ++s) {
                uint32_t const o = (uint32_t)ci->pairs[s].i;
                if (same_set && o == i) continue;
                nbr c;
                c.index = o;
                c.vector_to = sub(other[o], pos);
                c.distance = length(c.vector_to);
                if (c.distance >= max_distance) continue;
                list[cnt++] = c;
            }
        }
    }
    for (int a = 1; a < cnt; ++a) { /* insertion sort by neighbor_order */
        nbr const c = list[a];
        int b = a - 1;
        while (b >= 0 && nbr_less(&c, &list[b])) {
            list[b + 1] = list[b];
            --b;
        }
        list[b + 1] = c;
    }
    out->counts[i] = (uint8_t)cnt;
    for (int a = 0; a < cnt; ++a) {
        out->idx[i * NMAX + a] = list[a].index;
        out->dist[i * NMAX + a] = list[a].distance;
        out->vec[i * NMAX + a] = list[a].vector_to;
    }
}

static void build_all(v2 const* self,
                      size_t n,
                      v2 const* other,
                      int same_set,
                      cell_index const* ci,
                      float cell,
                      nbhd* out) {
    long long const nn = (long long)n;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < nn; ++i) build_one((size_t)i, self, other, same_set, ci, cell, cell, out);
}

/* compute_neighbor_kernels / compute_neighbor_kernel_gradients,
 * emerald/sph_common/neighborhood.cpp:178-210 */
static void nbhd_kernels(nbhd* nb, float support) {
    long long const nn = (long long)nb->n;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < nn; ++i) {
        for (int a = 0; a < nb->counts[i]; ++a) {
            size_t const o = (size_t)i * NMAX + a;
            nb->w[o] = kw(nb->dist[o], support);
            nb->gw[o] = kgradw(neg(nb->vec[o]), support);
        }
    }
}

/* compute_neighbor_distances_and_vectors_to,
 * emerald/sph_common/neighborhood.cpp:154-176 */
static void nbhd_recompute(nbhd* nb, v2 const* self, v2 const* other) {
    long long const nn = (long long)nb->n;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < nn; ++i) {
        for (int a = 0; a < nb->counts[i]; ++a) {
            size_t const o = (size_t)i * NMAX + a;
            v2 const d = sub(other[nb->idx[o]], self[i]);
            nb->vec[o] = d;
            nb->dist[o] = length(d);
        }
    }
}

void oracle_neighborhoods(float const* self_xy,
                          size_t n,
                          float const* other_xy,
                          size_t m,
                          int same_set,
                          float cell_size,
                          uint8_t* counts,
                          uint32_t* idx,
                          float* dist,
                          float* vec) {
    cell_index ci;
    cell_index_build(&ci, (v2 const*)other_xy, m, cell_size);
    nbhd nb;
    nbhd_alloc(&nb, n);
    build_all((v2 const*)self_xy, n, (v2 const*)other_xy, same_set, &ci, cell_size, &nb);
    for (size_t i = 0; i < n; ++i) {
        if (counts) counts[i] = nb.counts[i];
        for (int a = 0; a < NMAX; ++a) {
            size_t const o = i * NMAX + a;
            int const live = a < nb.counts[i];
            if (idx) idx[o] = live ? nb.idx[o] : 0u;
            if (dist) dist[o] = live ? nb.dist[o] : 0.0f;
            if (vec) {
                vec[2 * o] = live ? nb.vec[o].x : 0.0f;
                vec[2 * o + 1] = live ? nb.vec[o].y : 0.0f;
            }
        }
    }
    nbhd_free(&nb);
    cell_index_free(&ci);
}

/* compute_volumes, emerald/sph2d_box/solids.cpp:52-74 (with the neighbour
 * data of compute_neighbor_data_and_volumes, :76-137). */
void oracle_solid_volumes(float const* xy, size_t n, float support, float numer, float* volumes) {
    float const cell = support * 2.0f;
    cell_index ci;
    cell_index_build(&ci, (v2 const*)xy, n, cell);
    nbhd nb;
    nbhd_alloc(&nb, n);
    build_all((v2 const*)xy, n, (v2 const*)xy, 1, &ci, cell, &nb);
    float const w0 = kw(0.0f, support);
    for (size_t i = 0; i < n; ++i) {
        if (!nb.counts[i]) {
            volumes[i] = 1.0f / w0;
            continue;
        }
        float m = w0;
        for (int a = 0; a < nb.counts[i]; ++a) m += kw(nb.dist[i * NMAX + a], support);
        volumes[i] = numer / m;
    }
    nbhd_free(&nb);
    cell_index_free(&ci);
}

/* ------------------------------------------------------------- simulation */

struct oracle_sim {
    oracle_params p;
    size_t n;
    size_t ns;
    v2* x;
    v2* v;
    v2* xs;
    v2* vs;
    float* vol_s;
    int64_t time;
    cell_index solid_ci;
    nbhd fl;
    nbhd sl;
    /* Temp_data (emerald/sph2d_box/state.h:34-69) */
    v2* ext_forces;
    float* pressures;
    float* new_pressures;
    v2* pressure_forces;
    float* densities;
    v2* velocity_ext;
    v2* position_stars;
    v2* velocity_stars;
    float* alphas;
    float* div_kappas;
    float* dens_kappas;
    float* density_stars;
    float* aiis;
    v2* diis;
    v2* sum_dij_pjs;
    float* fluid_volumes;
    v2* pressure_accels;
};

void oracle_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n < 1 ? 1 : n);
#else
    (void)n;
#endif
}

#define ALLOCF(k) (float*)calloc((k) ? (k) : 1, sizeof(float))
#define ALLOCV(k) (v2*)calloc((k) ? (k) : 1, sizeof(v2))

oracle_sim* oracle_sim_create(oracle_params const* params,
                              float const* solid_xy,
                              float const* solid_volumes,
                              size_t n_solid,
                              float const* fluid_xy,
                              float const* fluid_v,
                              size_t n_fluid) {
    oracle_sim* s = (oracle_sim*)calloc(1, sizeof(oracle_sim));
    s->p = *params;
    s->n = n_fluid;
    s->ns = n_solid;
    s->x = ALLOCV(n_fluid);
    s->v = ALLOCV(n_fluid);
    memcpy(s->x, fluid_xy, n_fluid * sizeof(v2));
    if (fluid_v) memcpy(s->v, fluid_v, n_fluid * sizeof(v2));
    s->xs = ALLOCV(n_solid);
    s->vs = ALLOCV(n_solid);
    s->vol_s = ALLOCF(n_solid);
    memcpy(s->xs, solid_xy, n_solid * sizeof(v2));
    if (solid_volumes) {
        memcpy(s->vol_s, solid_volumes, n_solid * sizeof(float));
    } else {
        oracle_solid_volumes(solid_xy, n_solid, s->p.support, 1.7f, s->vol_s);
    }
    cell_index_build(&s->solid_ci, s->xs, n_solid, s->p.support * 2.0f);
    nbhd_alloc(&s->fl, n_fluid);
    nbhd_alloc(&s->sl, n_fluid);
    size_t const n = n_fluid;
    s->ext_forces = ALLOCV(n);
    s->pressures = ALLOCF(n);
    s->new_pressures = ALLOCF(n);
    s->pressure_forces = ALLOCV(n);
    s->densities = ALLOCF(n);
    s->velocity_ext = ALLOCV(n);
    s->position_stars = ALLOCV(n);
    s->velocity_stars = ALLOCV(n);
    s->alphas = ALLOCF(n);
    s->div_kappas = ALLOCF(n);
    s->dens_kappas = ALLOCF(n);
    s->density_stars = ALLOCF(n);
    s->aiis = ALLOCF(n);
    s->diis = ALLOCV(n);
    s->sum_dij_pjs = ALLOCV(n);
    s->fluid_volumes = ALLOCF(n);
    s->pressure_accels = ALLOCV(n);
    return s;
}

void oracle_sim_destroy(oracle_sim* s) {
    if (!s) return;
    free(s->x);
    free(s->v);
    free(s->xs);
    free(s->vs);
    free(s->vol_s);
    cell_index_free(&s->solid_ci);
    nbhd_free(&s->fl);
    nbhd_free(&s->sl);
    free(s->ext_forces);
    free(s->pressures);
    free(s->new_pressures);
    free(s->pressure_forces);
    free(s->densities);
    free(s->velocity_ext);
    free(s->position_stars);
    free(s->velocity_stars);
    free(s->alphas);
    free(s->div_kappas);
    free(s->dens_kappas);
    free(s->density_stars);
    free(s->aiis);
    free(s->diis);
    free(s->sum_dij_pjs);
    free(s->fluid_volumes);
    free(s->pressure_accels);
    free(s);
}

#define FOR_EACH(i, n)                          \
    _Pragma("omp parallel for schedule(static)") \
    for (long long i = 0; i < (long long)(n); ++i)

/* compute_all_neighbhorhoods, emerald/sph2d_box/neighborhoods_from_state.cpp:9-67 */
static void all_neighborhoods(oracle_sim* s) {
    float const cell = s->p.support * 2.0f;
    cell_index ci;
    cell_index_build(&ci, s->x, s->n, cell);
    build_all(s->x, s->n, s->x, 1, &ci, cell, &s->fl);
    build_all(s->x, s->n, s->xs, 0, &s->solid_ci, cell, &s->sl);
    cell_index_free(&ci);
}

/* compute_all_neighborhood_kernels, neighborhoods_from_state.cpp:69-101 */
static void all_kernels(oracle_sim* s) {
    nbhd_kernels(&s->fl, s->p.support);
    nbhd_kernels(&s->sl, s->p.support);
}

/* compute_all_external_forces + default_gravity_forces,
 * emerald/sph2d_box/forces.cpp:11-61, :63-83 */
static void external_forces(oracle_sim* s) {
    float const m = s->p.mass_per_particle;
    float const g = s->p.gravity;
    FOR_EACH(i, s->n) {
        s->ext_forces[i] = mk(0.0f, 0.0f);
        s->ext_forces[i].y -= m * g;
    }
}

/* compute_densities, emerald/sph_common/density.cpp:10-73 */
static void densities(oracle_sim* s) {
    float const rho0 = s->p.target_density;
    float const w0 = kw(0.0f, s->p.support);
    FOR_EACH(i, s->n) {
        float d = s->fluid_volumes[i] * rho0 * w0;
        int const c = s->fl.counts[i];
        for (int a = 0; a < c; ++a) {
            size_t const o = (size_t)i * NMAX + a;
            float const mass = rho0 * s->fluid_volumes[s->fl.idx[o]];
            d += s->fl.w[o] * mass;
        }
        s->densities[i] = d;
        int const cs = s->sl.counts[i];
        if (!cs) continue;
        float db = 0.0f;
        for (int a = 0; a < cs; ++a) {
            size_t const o = (size_t)i * NMAX + a;
            float const mass = rho0 * s->vol_s[s->sl.idx[o]];
            db += s->sl.w[o] * mass;
        }
        s->densities[i] += db;
    }
}

/* compute_divergences, emerald/sph_common/divergence.cpp:5-74 */
static void divergences(oracle_sim* s, float* out) {
    float const rho0 = s->p.target_density;
    FOR_EACH(i, s->n) {
        v2 const vi = s->v[i];
        int const c = s->fl.counts[i];
        if (!c) {
            out[i] = 0.0f;
        } else {
            float d = 0.0f;
            for (int a = 0; a < c; ++a) {
                size_t const o = (size_t)i * NMAX + a;
                uint32_t const j = s->fl.idx[o];
                float const mass = rho0 * s->fluid_volumes[j];
                d += mass * dot(sub(vi, s->v[j]), s->fl.gw[o]);
            }
            out[i] = d;
        }
        int const cs = s->sl.counts[i];
        if (!cs) continue;
        float db = 0.0f;
        for (int a = 0; a < cs; ++a) {
            size_t const o = (size_t)i * NMAX + a;
            uint32_t const j = s->sl.idx[o];
            float const mass = rho0 * s->vol_s[j];
            db += mass * dot(sub(vi, s->vs[j]), s->sl.gw[o]);
        }
        out[i] += db;
    }
}

/* predict_density_stars, emerald/sph_common/density.cpp:75-109 */
static void predict_density_stars(oracle_sim* s, float dt) {
    divergences(s, s->density_stars);
    FOR_EACH(i, s->n) {
        s->density_stars[i] = max_0x(s->densities[i] + (dt * s->density_stars[i]));
    }
}

static inline float p_over_rho2(float p, float rho) {
    float const d = sqrf(rho);
    return safe_f(p, d) ? p / d : 0.0f;
}

/* apply_pressures_in_place, emerald/sph_common/pressure.cpp:9-80 */
static void apply_pressures(oracle_sim* s, float dt, float const* p) {
    float const rho0 = s->p.target_density;
    FOR_EACH(i, s->n) {
        float const pi = p_over_rho2(p[i], s->densities[i]);
        int const c = s->fl.counts[i];
        if (c) {
            v2 acc = mk(0.0f, 0.0f);
            for (int a = 0; a < c; ++a) {
                size_t const o = (size_t)i * NMAX + a;
                uint32_t const j = s->fl.idx[o];
                float const mass = rho0 * s->fluid_volumes[j];
                float const pj = p_over_rho2(p[j], s->densities[j]);
                acc = add(acc, scl(-mass * (pi + pj), s->fl.gw[o]));
            }
            s->v[i] = add(s->v[i], scl(dt, acc));
        }
        int const cs = s->sl.counts[i];
        if (cs) {
            v2 acc = mk(0.0f, 0.0f);
            for (int a = 0; a < cs; ++a) {
                size_t const o = (size_t)i * NMAX + a;
                float const mass = rho0 * s->vol_s[s->sl.idx[o]];
                acc = add(acc, scl(-mass * pi, s->sl.gw[o]));
            }
            s->v[i] = add(s->v[i], scl(dt, acc));
        }
    }
}

/* compute_pressure_accelerations, emerald/sph_common/pressure.cpp:83-178
 * (also iisph_pseudo_ap_compute_pseudo_pressure_displacements,
 * emerald/sph2d_box/iisph_pseudo_ap_ops.cpp:119-224, the same sum). */
static void pressure_accelerations(oracle_sim* s, float const* p, v2* out) {
    float const rho0 = s->p.target_density;
    FOR_EACH(i, s->n) {
        float const pi = p_over_rho2(p[i], s->densities[i]);
        int const c = s->fl.counts[i];
        if (!c) {
            out[i] = mk(0.0f, 0.0f);
        } else {
            v2 acc = mk(0.0f, 0.0f);
            for (int a = 0; a < c; ++a) {
                size_t const o = (size_t)i * NMAX + a;
                uint32_t const j = s->fl.idx[o];
                float const mass = rho0 * s->fluid_volumes[j];
                float const coeff = pi + p_over_rho2(p[j], s->densities[j]);
                acc = add(acc, scl(-mass * coeff, s->fl.gw[o]));
            }
            out[i] = acc;
        }
        int const cs = s->sl.counts[i];
        if (!cs) continue;
        v2 acc = mk(0.0f, 0.0f);
        for (int a = 0; a < cs; ++a) {
            size_t const o = (size_t)i * NMAX + a;
            float const mass = rho0 * s->vol_s[s->sl.idx[o]];
            acc = add(acc, scl(-mass * pi, s->sl.gw[o]));
        }
        out[i] = add(out[i], acc);
    }
}

/* integrate_velocities_in_place (forces), emerald/sph_common/dynamics.cpp:24-37 */
static void integrate_velocities_ext(oracle_sim* s, float dt) {
    float const rho0 = s->p.target_density;
    FOR_EACH(i, s->n) {
        float const denom = rho0 * s->fluid_volumes[i];
        v2 const numer = scl(dt, s->ext_forces[i]);
        if (safe_v(numer, denom)) s->v[i] = add(s->v[i], divs(numer, denom));
    }
}

/* integrate_positions_in_place, emerald/sph_common/dynamics.cpp:46-51 */
static void integrate_positions(oracle_sim* s, float dt) {
    FOR_EACH(i, s->n) { s->x[i] = add(s->x[i], scl(dt, s->v[i])); }
}

/* compute_constant_volumes, emerald/sph_common/volume.cpp:7-14 */
static void constant_volumes(oracle_sim* s) {
    float const vol = s->p.mass_per_particle / s->p.target_density;
    for (size_t i = 0; i < s->n; ++i) s->fluid_volumes[i] = vol;
}

/* Error accumulation of iisph_compute_new_pressures and the AP variants:
 * sum of uint64(error * 1000) and the maximum
 * (emerald/sph2d_box/iisph_ops.cpp:411-424). */
static void pack_error(uint64_t sum, float mx, size_t n, float* avg, float* max) {
    double const numer = (double)sum;
    double const denom = (double)(1000 * n);
    *avg = (float)(numer / denom);
    *max = mx;
}

/* ---- IISPH, emerald/sph2d_box/iisph_ops.cpp and iisph.cpp:23-151 ---- */

static void iisph_diis(oracle_sim* s, float dt) {
    float const rho0 = s->p.target_density;
    FOR_EACH(i, s->n) {
        float const rho = s->densities[i];
        int const c = s->fl.counts[i];
        if (!c) {
            s->diis[i] = mk(0.0f, 0.0f);
        } else {
            v2 g = mk(0.0f, 0.0f);
            for (int a = 0; a < c; ++a) {
                size_t const o = (size_t)i * NMAX + a;
                float const mass = rho0 * s->fluid_volumes[s->fl.idx[o]];
                g = add(g, scl(mass, s->fl.gw[o]));
            }
            v2 const numer = scl(-sqrf(dt), g);
            float const denom = sqrf(rho);
            s->diis[i] = safe_v(numer, denom) ? divs(numer, denom) : mk(0.0f, 0.0f);
        }
        int const cs = s->sl.counts[i];
        if (!cs) continue;
        v2 g = mk(0.0f, 0.0f);
        for (int a = 0; a < cs; ++a) {
            size_t const o = (size_t)i * NMAX + a;
            float const mass = rho0 * s->vol_s[s->sl.idx[o]];
            g = add(g, scl(mass, s->sl.gw[o]));
        }
        v2 const numer = scl(-sqrf(dt), g);
        float const denom = sqrf(rho);
        s->diis[i] = add(s->diis[i], safe_v(numer, denom) ? divs(numer, denom) : mk(0.0f, 0.0f));
    }
}

static void iisph_aiis_and_density_stars(oracle_sim* s, float dt) {
    float const rho0 = s->p.target_density;
    FOR_EACH(i, s->n) {
        v2 const dii = s->diis[i];
        v2 const vi = s->v[i];
        int const c = s->fl.counts[i];
        if (!c) {
            s->density_stars[i] = s->densities[i];
            s->aiis[i] = 0.0f;
        } else {
            float aii = 0.0f;
            float dd = 0.0f;
            for (int a = 0; a < c; ++a) {
                size_t const o = (size_t)i * NMAX + a;
                uint32_t const j = s->fl.idx[o];
                v2 const gw = s->fl.gw[o];
                float const mass = s->fluid_volumes[j] * rho0;
                v2 const numer = scl(-sqrf(dt) * mass, gw);
                float const denom = sqrf(s->densities[j]);
                if (safe_v(numer, denom)) {
                    v2 const dij = divs(numer, denom);
                    v2 const dji = neg(dij);
                    aii += mass * dot(sub(dii, dji), gw);
                }
                dd += dt * mass * dot(sub(vi, s->v[j]), gw);
            }
            s->aiis[i] = aii;
            s->density_stars[i] = s->densities[i] + dd;
        }
        int const cs = s->sl.counts[i];
        if (!cs) continue;
        float aii = 0.0f;
        float dd = 0.0f;
        for (int a = 0; a < cs; ++a) {
            size_t const o = (size_t)i * NMAX + a;
            uint32_t const j = s->sl.idx[o];
            v2 const gw = s->sl.gw[o];
            float const mass = s->vol_s[j] * rho0;
            aii += mass * dot(dii, gw);
            dd += dt * mass * dot(sub(vi, s->vs[j]), gw);
        }
        s->aiis[i] += aii;
        s->density_stars[i] += dd;
    }
}

static void iisph_sum_dij_pjs(oracle_sim* s, float dt) {
    float const rho0 = s->p.target_density;
    float const* p = s->pressures;
    FOR_EACH(i, s->n) {
        int const c = s->fl.counts[i];
        v2 sum = mk(0.0f, 0.0f);
        for (int a = 0; a < c; ++a) {
            size_t const o = (size_t)i * NMAX + a;
            uint32_t const j = s->fl.idx[o];
            float const mass = s->fluid_volumes[j] * rho0;
            v2 const numer = scl(-sqrf(dt) * mass * p[j], s->fl.gw[o]);
            float const denom = sqrf(s->densities[j]);
            if (safe_v(numer, denom)) sum = add(sum, divs(numer, denom));
        }
        s->sum_dij_pjs[i] = sum;
    }
}

static void iisph_betas(oracle_sim* s, float dt, float* betas) {
    float const rho0 = s->p.target_density;
    float const* p = s->pressures;
    FOR_EACH(i, s->n) {
        float const pi = p[i];
        v2 const si = s->sum_dij_pjs[i];
        int const c = s->fl.counts[i];
        if (!c) {
            betas[i] = 0.0f;
        } else {
            float beta = 0.0f;
            for (int a = 0; a < c; ++a) {
                size_t const o = (size_t)i * NMAX + a;
                uint32_t const j = s->fl.idx[o];
                v2 const gw = s->fl.gw[o];
                float const mass = rho0 * s->fluid_volumes[j];
                v2 const numer = scl(-sqrf(dt) * mass, gw);
                float const denom = sqrf(s->densities[j]);
                v2 const dij = safe_v(numer, denom) ? divs(numer, denom) : mk(0.0f, 0.0f);
                v2 const dji = neg(dij);
                v2 const sknoti = sub(s->sum_dij_pjs[j], scl(pi, dji));
                v2 const t = sub(sub(si, scl(p[j], s->diis[j])), sknoti);
                beta += mass * dot(t, gw);
            }
            betas[i] = beta;
        }
        int const cs = s->sl.counts[i];
        if (!cs) continue;
        float beta = 0.0f;
        for (int a = 0; a < cs; ++a) {
            size_t const o = (size_t)i * NMAX + a;
            float const mass = rho0 * s->vol_s[s->sl.idx[o]];
            beta += mass * dot(si, s->sl.gw[o]);
        }
        betas[i] += beta;
    }
}

static void iisph_new_pressures(oracle_sim* s, float* io, float* avg, float* max) {
    float const rho0 = s->p.target_density;
    float const omega = s->p.iisph_omega;
    uint64_t sum = 0;
    float mx = 0.0f;
#pragma omp parallel for schedule(static) reduction(+ : sum) reduction(max : mx)
    for (long long i = 0; i < (long long)s->n; ++i) {
        float const alpha = s->aiis[i];
        float const old = s->pressures[i];
        if (alpha == 0.0f) {
            io[i] = old;
            continue;
        }
        float const numer = rho0 - s->density_stars[i] - io[i];
        if (!safe_f(numer, alpha)) {
            io[i] = old;
            continue;
        }
        float const err = max_0x(-(numer - (alpha * old)) / rho0);
        if (mx < err) mx = err;
        sum += (uint64_t)(err * 1000.0f);
        io[i] = max_0x(mix(old, numer / alpha, omega));
    }
    pack_error(sum, mx, s->n, avg, max);
}

static void iisph_sub_step(oracle_sim* s, float dt, oracle_stats* st) {
    all_neighborhoods(s);
    all_kernels(s);
    external_forces(s);
    densities(s);
    integrate_velocities_ext(s, dt);
    iisph_diis(s, dt);
    iisph_aiis_and_density_stars(s, dt);
    memset(s->pressures, 0, s->n * sizeof(float));
    int iter = 0;
    float avg = 0.0f, mx = 0.0f;
    for (; iter < s->p.iisph_max_pressure_iterations; ++iter) {
        iisph_sum_dij_pjs(s, dt);
        iisph_betas(s, dt, s->new_pressures);
        iisph_new_pressures(s, s->new_pressures, &avg, &mx);
        float* t = s->pressures;
        s->pressures = s->new_pressures;
        s->new_pressures = t;
        if (iter > 1 && avg <= s->p.iisph_error_average_threshold &&
            mx <= s->p.iisph_error_max_threshold) {
            break;
        }
    }
    if (st) {
        st->pressure_iterations = iter < s->p.iisph_max_pressure_iterations ? iter + 1 : iter;
        st->error_average = avg;
        st->error_max = mx;
    }
    apply_pressures(s, dt, s->pressures);
    integrate_positions(s, dt);
}

/* ---- IISPH_AP, emerald/sph2d_box/iisph_ap_ops.cpp, iisph_ap.cpp:44-154 ---- */

static void ap_density_stars_and_diagonals(oracle_sim* s, float dt, int pseudo) {
    float const rho0 = s->p.target_density;
    FOR_EACH(i, s->n) {
        int const c = s->fl.counts[i];
        int const cs = s->sl.counts[i];
        if (!(c + cs)) {
            s->density_stars[i] = s->densities[i];
            s->aiis[i] = 0.0f;
            continue;
        }
        float const self_mass = s->fluid_volumes[i] * rho0;
        float const rho = s->densities[i];
        v2 const vi = s->v[i];
        v2 sum = mk(0.0f, 0.0f);
        float sdot = 0.0f;
        float div = 0.0f;
        for (int a = 0; a < c; ++a) {
            size_t const o = (size_t)i * NMAX + a;
            uint32_t const j = s->fl.idx[o];
            v2 const gw = s->fl.gw[o];
            float const mass = s->fluid_volumes[j] * rho0;
            sum = add(sum, scl(mass, gw));
            sdot += mass * dot(gw, gw);
            div += mass * dot(sub(vi, s->v[j]), gw);
        }
        for (int a = 0; a < cs; ++a) {
            size_t const o = (size_t)i * NMAX + a;
            uint32_t const j = s->sl.idx[o];
            v2 const gw = s->sl.gw[o];
            float const mass = s->vol_s[j] * rho0;
            sum = add(sum, scl(mass, gw));
            div += mass * dot(sub(vi, s->vs[j]), gw);
        }
        float const denom = sqrf(rho);
        float numer;
        if (pseudo) {
            numer = -(dot(sum, sum) + self_mass * sdot);
        } else {
            numer = -sqrf(dt) * (dot(sum, sum) + self_mass * sdot);
        }
        s->aiis[i] = safe_f(numer, denom) ? numer / denom : 0.0f;
        s->density_stars[i] = rho + dt * div;
    }
}

static void ap_iterate(oracle_sim* s, float dt, int pseudo, float* avg, float* max) {
    float const rho0 = s->p.target_density;
    float const omega = s->p.iisph_omega;
    uint64_t sum = 0;
    float mx = 0.0f;
#pragma omp parallel for schedule(static) reduction(+ : sum) reduction(max : mx)
    for (long long i = 0; i < (long long)s->n; ++i) {
        int const c = s->fl.counts[i];
        int const cs = s->sl.counts[i];
        if (!c && !cs) {
            s->pressures[i] = 0.0f;
            continue;
        }
        float const diag = s->aiis[i];
        if (pseudo && diag == 0.0f) {
            s->pressures[i] = 0.0f;
            continue;
        }
        float api = 0.0f;
        v2 const ai = s->pressure_accels[i];
        for (int a = 0; a < c; ++a) {
            size_t const o = (size_t)i * NMAX + a;
            uint32_t const j = s->fl.idx[o];
            float const mass = rho0 * s->fluid_volumes[j];
            api += mass * dot(sub(ai, s->pressure_accels[j]), s->fl.gw[o]);
        }
        for (int a = 0; a < cs; ++a) {
            size_t const o = (size_t)i * NMAX + a;
            float const mass = rho0 * s->vol_s[s->sl.idx[o]];
            api += mass * dot(ai, s->sl.gw[o]);
        }
        if (!pseudo) api *= sqrf(dt);
        float const source = rho0 - s->density_stars[i];
        float const r = api - source;
        float const err = max_0x(safe_f(r, rho0) ? r / rho0 : 0.0f);
        if (mx < err) mx = err;
        sum += (uint64_t)(err * 1000.0f);
        float const old = s->pressures[i];
        float const numer = omega * (source - api);
        s->pressures[i] = max_0x(old + (safe_f(numer, diag) ? numer / diag : 0.0f));
    }
    pack_error(sum, mx, s->n, avg, max);
}

static void ap_sub_step(oracle_sim* s, float dt, int pseudo, oracle_stats* st) {
    all_neighborhoods(s);
    all_kernels(s);
    external_forces(s);
    densities(s);
    integrate_velocities_ext(s, dt);
    ap_density_stars_and_diagonals(s, dt, pseudo);
    memset(s->pressures, 0, s->n * sizeof(float));
    int iter = 0;
    float avg = 0.0f, mx = 0.0f;
    for (; iter < s->p.iisph_max_pressure_iterations; ++iter) {
        pressure_accelerations(s, s->pressures, s->pressure_accels);
        ap_iterate(s, dt, pseudo, &avg, &mx);
        if (iter > 1 && avg <= s->p.iisph_error_average_threshold &&
            mx <= s->p.iisph_error_max_threshold) {
            break;
        }
    }
    if (st) {
        st->pressure_iterations = iter < s->p.iisph_max_pressure_iterations ? iter + 1 : iter;
        st->error_average = avg;
        st->error_max = mx;
    }
    pressure_accelerations(s, s->pressures, s->pressure_accels);
    if (!pseudo) {
        /* integrate_velocities_and_positions_in_place, dynamics.cpp:53-63 */
        FOR_EACH(i, s->n) {
            s->v[i] = add(s->v[i], scl(dt, s->pressure_accels[i]));
            s->x[i] = add(s->x[i], scl(dt, s->v[i]));
        }
    } else {
        /* iisph_pseudo_ap_integrate_velocities_and_positions_in_place,
         * iisph_pseudo_ap_ops.cpp:325-343 */
        FOR_EACH(i, s->n) {
            v2 const vstar = s->v[i];
            v2 const disp = s->pressure_accels[i];
            s->x[i] = add(add(s->x[i], scl(dt, vstar)), disp);
            if (safe_v(vstar, dt)) s->v[i] = add(vstar, divs(disp, dt));
        }
    }
}

/* ---- DFSPH_P, emerald/sph2d_box/dfsph_p_ops.cpp, dfsph_p.cpp:61-374 ---- */

static void dfsph_alphas(oracle_sim* s) {
    float const rho0 = s->p.target_density;
    FOR_EACH(i, s->n) {
        int const c = s->fl.counts[i];
        int const cs = s->sl.counts[i];
        if (!(c + cs)) {
            s->alphas[i] = 0.0f;
            continue;
        }
        v2 sum = mk(0.0f, 0.0f);
        float sdot = 0.0f;
        for (int a = 0; a < c; ++a) {
            size_t const o = (size_t)i * NMAX + a;
            v2 const m = scl(s->fluid_volumes[s->fl.idx[o]] * rho0, s->fl.gw[o]);
            sum = add(sum, m);
            sdot += dot(m, m);
        }
        for (int a = 0; a < cs; ++a) {
            size_t const o = (size_t)i * NMAX + a;
            sum = add(sum, scl(s->vol_s[s->sl.idx[o]] * rho0, s->sl.gw[o]));
        }
        float const numer = sqrf(s->densities[i]);
        float const denom = dot(sum, sum) + sdot;
        s->alphas[i] = safe_f(numer, denom) ? numer / denom : 0.0f;
    }
}

/* compute_transformed_scalar_average_and_max, emerald/sph_common/common.h:209-232 */
static void transformed_avg_max(oracle_sim* s, float dt, int divergence, float* avg, float* max) {
    float const rho0 = s->p.target_density;
    int64_t sum = 0;
    float mx = -FLT_MAX;
#pragma omp parallel for schedule(static) reduction(+ : sum) reduction(max : mx)
    for (long long i = 0; i < (long long)s->n; ++i) {
        float const val = s->density_stars[i];
        float e;
        if (divergence) {
            e = val <= 0.0f ? 0.0f : (dt * val / rho0);
        } else {
            float const err = val - rho0;
            e = err <= 0.0f ? 0.0f : (err / rho0);
        }
        if (mx < e) mx = e;
        sum += (int64_t)(e * 1000.0f);
    }
    if (s->n < 1) {
        *avg = 0.0f;
        *max = 0.0f;
        return;
    }
    *avg = (float)((double)sum / (double)(1000 * s->n));
    *max = mx;
}

static void dfsph_correct_divergence(oracle_sim* s, float dt, oracle_stats* st) {
    apply_pressures(s, dt, s->div_kappas);
    int iter = 0;
    float avg = 0.0f, mx = 0.0f;
    for (; iter < s->p.dfsph_max_correction_iterations; ++iter) {
        divergences(s, s->density_stars);
        FOR_EACH(i, s->n) {
            float const d = s->density_stars[i];
            if (d <= 0.0f) {
                s->div_kappas[i] = 0.0f;
            } else {
                float const numer = d * s->alphas[i];
                s->div_kappas[i] = safe_f(numer, dt) ? numer / dt : 0.0f;
            }
        }
        apply_pressures(s, dt, s->div_kappas);
        if (iter > 0) {
            transformed_avg_max(s, dt, 1, &avg, &mx);
            if (avg <= s->p.dfsph_divergence_error_average_threshold &&
                mx <= s->p.dfsph_divergence_error_max_threshold) {
                break;
            }
        }
    }
    if (st) {
        st->divergence_iterations = iter < s->p.dfsph_max_correction_iterations ? iter + 1 : iter;
        st->divergence_error_average = avg;
        st->divergence_error_max = mx;
    }
}

static void dfsph_correct_density(oracle_sim* s, float dt, oracle_stats* st) {
    float const rho0 = s->p.target_density;
    apply_pressures(s, dt, s->dens_kappas);
    int iter = 0;
    float avg = 0.0f, mx = 0.0f;
    for (; iter < s->p.dfsph_max_correction_iterations; ++iter) {
        predict_density_stars(s, dt);
        FOR_EACH(i, s->n) {
            float const delta = s->density_stars[i] - rho0;
            if (delta <= 0.0f) {
                s->dens_kappas[i] = 0.0f;
            } else {
                float const numer = delta * s->alphas[i];
                float const d = sqrf(dt);
                s->dens_kappas[i] = safe_f(numer, d) ? numer / d : 0.0f;
            }
        }
        apply_pressures(s, dt, s->dens_kappas);
        if (iter > 1) {
            transformed_avg_max(s, dt, 0, &avg, &mx);
            if (avg <= s->p.dfsph_density_error_average_threshold &&
                mx <= s->p.dfsph_density_error_max_threshold) {
                break;
            }
        }
    }
    if (st) {
        st->pressure_iterations = iter < s->p.dfsph_max_correction_iterations ? iter + 1 : iter;
        st->error_average = avg;
        st->error_max = mx;
    }
}

static void dfsph_sub_step(oracle_sim* s, float dt, oracle_stats* st) {
    all_neighborhoods(s);
    all_kernels(s);
    densities(s);
    dfsph_alphas(s);
    dfsph_correct_divergence(s, dt, st);
    external_forces(s);
    integrate_velocities_ext(s, dt);
    dfsph_correct_density(s, dt, st);
    integrate_positions(s, dt);
}

/* ---- PCISPH, emerald/sph2d_box/pcisph_ops.cpp, pcisph.cpp:36-164 ---- */

static void pcisph_sub_step(oracle_sim* s, float dt, oracle_stats* st) {
    float const m = s->p.mass_per_particle;
    float const rho0 = s->p.target_density;
    float const h = s->p.support;
    float const visc = s->p.viscosity;
    float const w0 = kw(0.0f, h);
    all_neighborhoods(s);
    external_forces(s);
    float const mult = dt / m;
    FOR_EACH(i, s->n) {
        s->velocity_ext[i] = s->v[i];
        s->velocity_ext[i] = add(s->velocity_ext[i], scl(mult, s->ext_forces[i]));
    }
    memset(s->pressures, 0, s->n * sizeof(float));
    int pass = 0;
    float max_err = 0.0f;
    for (; pass < 6; ++pass) {
        FOR_EACH(i, s->n) {
            v2 vs = s->velocity_ext[i];
            if (pass > 0) vs = add(vs, scl(mult, s->pressure_forces[i]));
            s->velocity_stars[i] = vs;
            s->position_stars[i] = add(s->x[i], scl(dt, vs));
        }
        nbhd_recompute(&s->fl, s->position_stars, s->position_stars);
        nbhd_recompute(&s->sl, s->position_stars, s->xs);
        all_kernels(s);
        FOR_EACH(i, s->n) {
            s->pressure_forces[i] = mk(0.0f, 0.0f);
            /* pcisph_compute_densities, pcisph_ops.cpp:18-38 */
            int const c = s->fl.counts[i];
            if (!c) {
                s->densities[i] = m * w0;
            } else {
                float ws = w0;
                for (int a = 0; a < c; ++a) ws += s->fl.w[(size_t)i * NMAX + a];
                s->densities[i] = m * ws;
            }
            /* pcisph_accumulate_density_from_solids, :40-63 */
            int const cs = s->sl.counts[i];
            if (cs) {
                float vf = 0.0f;
                for (int a = 0; a < cs; ++a) {
                    size_t const o = (size_t)i * NMAX + a;
                    vf += s->vol_s[s->sl.idx[o]] * s->sl.w[o];
                }
                s->densities[i] += rho0 * vf;
            }
            /* pcisph_update_pressures, :65-76 */
            float const err = max_x0(s->densities[i] - rho0);
            s->pressures[i] += err / s->p.pressure_correction_denom;
        }
        float const H = h;
        float const N2 = 0.01f * H * H;
        FOR_EACH(i, s->n) {
            /* pcisph_accumulate_pressure_forces, :78-142 */
            int const c = s->fl.counts[i];
            if (c) {
                v2 const vi = s->velocity_stars[i];
                float const rho = s->densities[i];
                float const pors = s->pressures[i] / sqrf(rho);
                v2 pf = mk(0.0f, 0.0f);
                for (int a = 0; a < c; ++a) {
                    size_t const o = (size_t)i * NMAX + a;
                    uint32_t const j = s->fl.idx[o];
                    v2 const vto = s->fl.vec[o];
                    v2 const gw = s->fl.gw[o];
                    float const rho_j = s->densities[j];
                    pf = add(pf, scl(pors + (s->pressures[j] / sqrf(rho_j)), gw));
                    v2 const dv = sub(s->velocity_stars[j], vi);
                    float const dvr = dot(vto, dv);
                    if (dvr < 0.0f) {
                        float const mu = H * dvr / (s->fl.dist[o] + N2);
                        float const den = (rho + rho_j) / 2.0f;
                        pf = add(pf, scl(((-1.0f * visc * mu) + (2.0f * sqrf(mu))) / den, gw));
                    }
                }
                s->pressure_forces[i] = add(s->pressure_forces[i], scl(-(m * m), pf));
            }
            /* pcisph_accumulate_pressure_forces_from_solids, :144-178 */
            int const cs = s->sl.counts[i];
            if (cs) {
                float const pors = s->pressures[i] / sqrf(s->densities[i]);
                v2 vg = mk(0.0f, 0.0f);
                for (int a = 0; a < cs; ++a) {
                    size_t const o = (size_t)i * NMAX + a;
                    vg = add(vg, scl(s->vol_s[s->sl.idx[o]], s->sl.gw[o]));
                }
                s->pressure_forces[i] = add(s->pressure_forces[i], scl(-m * rho0 * pors, vg));
            }
        }
        if (pass > 1) {
            /* max_density_error, emerald/sph_common/common.cpp:78-85 */
            float mx = 0.0f;
            for (size_t i = 0; i < s->n; ++i) {
                float const e = max_0x(s->densities[i] - rho0);
                if (mx < e) mx = e;
            }
            max_err = mx;
            if ((mx / rho0) <= 0.01f) break;
        }
    }
    if (st) {
        st->pressure_iterations = pass < 6 ? pass + 1 : pass;
        st->error_max = max_err / rho0;
        st->error_average = 0.0f;
    }
    FOR_EACH(i, s->n) {
        s->v[i] = s->velocity_ext[i];
        s->v[i] = add(s->v[i], scl(mult, s->pressure_forces[i]));
        s->x[i] = add(s->x[i], scl(dt, s->v[i]));
    }
}

/* ------------------------------------------------------ frame and access */

/* Per-frame initialisation of the solver temporaries: the kappa reset of
 * dfsph_p_resize_and_init_temp_arrays (emerald/sph2d_box/dfsph_p.cpp:214-229)
 * and compute_constant_volumes (adaptive_time_step.h:57-61). */
int oracle_sim_begin_frame(oracle_sim* s, int method) {
    if (method < 0 || method > 4) return -1;
    if (method == 4) {
        memset(s->div_kappas, 0, s->n * sizeof(float));
        memset(s->dens_kappas, 0, s->n * sizeof(float));
    }
    if (method != 0) constant_volumes(s);
    return 0;
}

int oracle_sim_sub_step(oracle_sim* s, int method, float t, float dt, oracle_stats* st) {
    (void)t;
    if (st) memset(st, 0, sizeof(*st));
    switch (method) {
    case 0: pcisph_sub_step(s, dt, st); return 0;
    case 1: iisph_sub_step(s, dt, st); return 0;
    case 2: ap_sub_step(s, dt, 0, st); return 0;
    case 3: ap_sub_step(s, dt, 1, st); return 0;
    case 4: dfsph_sub_step(s, dt, st); return 0;
    default: return -1;
    }
}

static double to_seconds(int64_t f) { return (double)f / FLICKS_PER_SECOND; }
static int64_t to_flicks(double sec) { return (int64_t)(sec * FLICKS_PER_SECOND); }

/* cfl_maximum_time_step, emerald/sph_common/cfl.cpp:12-21 */
static int64_t cfl_step(oracle_sim* s, float factor) {
    float mx = 0.0f;
    for (size_t i = 0; i < s->n; ++i) {
        float const d = dot(s->v[i], s->v[i]);
        if (mx < d) mx = d;
    }
    double const numer = factor * s->p.support;
    double const denom = sqrt((double)mx);
    double const r = safe_d(numer, denom) ? numer / denom : (double)1.0f;
    return to_flicks(r);
}

/* std_adaptive_time_step, emerald/sph2d_box/adaptive_time_step.h:35-122, and
 * pcisph_simulation_step, emerald/sph2d_box/pcisph.cpp:166-204. */
int oracle_sim_frame(oracle_sim* s, int method) {
    int64_t const tps = s->p.time_per_step_flicks;
    if (method == 0) {
        int64_t const per = tps / s->p.sub_steps;
        int64_t time = s->time;
        for (int k = 0; k < s->p.sub_steps; ++k) {
            pcisph_sub_step(s, s->p.seconds_per_sub_step, NULL);
            time += per;
        }
        s->time += tps;
        return s->p.sub_steps;
    }
    int min_denom = 60, max_denom = 4;
    float factor = 0.4f;
    if (method == 1) {
        max_denom = 6;
        factor = 0.2f;
    }
    if (oracle_sim_begin_frame(s, method)) return -1;
    int const divisor = min_denom / max_denom;
    int remaining = min_denom;
    int64_t const tpss = tps / remaining;
    int64_t time = s->time;
    int count = 0;
    while (remaining > 0) {
        int64_t const cfl = cfl_step(s, factor);
        int num = (int)ceil(to_seconds(cfl) / to_seconds(tpss));
        if (num < 1) num = 1;
        if (num > divisor) num = divisor;
        if (num > remaining) num = remaining;
        int64_t const sub_dt = num * tpss;
        oracle_sim_sub_step(s, method, (float)to_seconds(time), (float)to_seconds(sub_dt), NULL);
        remaining -= num;
        time += sub_dt;
        ++count;
    }
    s->time += tps;
    return count;
}

int64_t oracle_sim_time(oracle_sim const* s) { return s->time; }

void oracle_sim_get_state(oracle_sim const* s, float* x, float* v) {
    if (x) memcpy(x, s->x, s->n * sizeof(v2));
    if (v) memcpy(v, s->v, s->n * sizeof(v2));
}

void oracle_sim_set_state(oracle_sim* s, float const* x, float const* v) {
    if (x) memcpy(s->x, x, s->n * sizeof(v2));
    if (v) memcpy(s->v, v, s->n * sizeof(v2));
}

int oracle_sim_get_array(oracle_sim const* s, char const* name, float* out) {
    struct {
        char const* name;
        void const* data;
        int width;
    } const table[] = {
      {"densities", s->densities, 1},
      {"pressures", s->pressures, 1},
      {"new_pressures", s->new_pressures, 1},
      {"density_stars", s->density_stars, 1},
      {"aiis", s->aiis, 1},
      {"alphas", s->alphas, 1},
      {"divergence_kappas", s->div_kappas, 1},
      {"density_kappas", s->dens_kappas, 1},
      {"fluid_volumes", s->fluid_volumes, 1},
      {"diis", s->diis, 2},
      {"sum_dij_pjs", s->sum_dij_pjs, 2},
      {"external_forces", s->ext_forces, 2},
      {"pressure_forces", s->pressure_forces, 2},
      {"pressure_accelerations", s->pressure_accels, 2},
      {"velocity_external_forces", s->velocity_ext, 2},
      {"position_stars", s->position_stars, 2},
      {"velocity_stars", s->velocity_stars, 2},
      {"solid_volumes", s->vol_s, 1},
    };
    for (size_t k = 0; k < sizeof(table) / sizeof(table[0]); ++k) {
        if (strcmp(table[k].name, name) == 0) {
            size_t const count = (strcmp(name, "solid_volumes") == 0) ? s->ns : s->n;
            if (out) memcpy(out, table[k].data, count * table[k].width * sizeof(float));
            return table[k].width;
        }
    }
    return -1;
}

void oracle_sim_get_neighbors(oracle_sim const* s,
                              int solid,
                              uint8_t* counts,
                              uint32_t* idx,
                              float* w,
                              float* gw) {
    nbhd const* nb = solid ? &s->sl : &s->fl;
    for (size_t i = 0; i < s->n; ++i) {
        if (counts) counts[i] = nb->counts[i];
        for (int a = 0; a < NMAX; ++a) {
            size_t const o = i * NMAX + a;
            int const live = a < nb->counts[i];
            if (idx) idx[o] = live ? nb->idx[o] : 0u;
            if (w) w[o] = live ? nb->w[o] : 0.0f;
            if (gw) {
                gw[2 * o] = live ? nb->gw[o].x : 0.0f;
                gw[2 * o + 1] = live ? nb->gw[o].y : 0.0f;
            }
        }
    }
}
