// FP64 GPU oracle of the DFSPH_P, IISPH, IISPH_AP, IISPH_PSEUDO_AP and
// PCISPH sub-steps: test infrastructure only.
//
// The same formulas and neighbour-list order as the reference's sph_common
// and dfsph_p code (cubic spline W/GradW, emerald/sph_common/kernels.h:12-64;
// densities, emerald/sph_common/density.cpp:10-73; divergences,
// emerald/sph_common/divergence.cpp:5-74; apply_pressures_in_place,
// emerald/sph_common/pressure.cpp:9-80; DFSPH_P coefficients and pseudo
// pressures, emerald/sph2d_box/dfsph_p_ops.cpp:19-126; the sub-step order of
// emerald/sph2d_box/dfsph_p.cpp:325-373; the IISPH coefficients, pressure
// iteration and sub-step order of emerald/sph2d_box/iisph_ops.cpp:20-425
// and emerald/sph2d_box/iisph.cpp:23-151; the AP diagonal and Jacobi step of
// emerald/sph2d_box/iisph_ap_ops.cpp:19-194 and iisph_pseudo_ap_ops.cpp:19-343
// with the sub-step orders of iisph_ap.cpp:44-189 and
// iisph_pseudo_ap.cpp:64-194; the PCISPH predictor-corrector passes of
// emerald/sph2d_box/pcisph_ops.cpp:18-178 and pcisph.cpp:36-164, with the
// lists' distances and kernels recomputed at the predicted positions,
// neighborhoods_from_state.cpp:103-128), evaluated in double. It states the
// error of the FP32 results: the caller passes each sub-step's dt and the
// iteration counts the FP32 run took, so the two runs differ only in
// arithmetic precision.
//
// Independent of the product's kernels: neighbours come from a sort of
// (cell key, index) pairs and a binary search per cell, lists are built by
// sorted insertion on (distance, index), and every loop is a plain
// one-thread-per-particle kernel driven from the host.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>
#include <thrust/device_ptr.h>
#include <thrust/sort.h>

namespace {

constexpr int kMax = 64;
constexpr double kPi = 3.14159274101257324218750;  // the reference's float pi, widened

struct Params {
    double support, rho0, mass, fluid_volume, gravity;
};

struct Sim {
    Params p;
    size_t n = 0, ns = 0;
    double2 *x = nullptr, *v = nullptr, *xs = nullptr;
    double* vols = nullptr;
    double *rho = nullptr, *alpha = nullptr, *kdiv = nullptr, *kdens = nullptr, *qdiv = nullptr,
           *qdens = nullptr, *rho_star = nullptr, *div = nullptr;
    // IISPH: diagonal terms, pressures (current and next), sum_j dij pj
    double2 *dii = nullptr, *sdp = nullptr;
    double *aii = nullptr, *pres = nullptr, *pres_next = nullptr;
    // PCISPH: velocity after external forces, predicted velocity and
    // position, pressure force; AP: pressure accelerations (displacements)
    double2 *vext = nullptr, *vstar = nullptr, *xstar = nullptr, *fpres = nullptr, *acc = nullptr;
    // neighbour lists, slot-major: entry k of particle i at k * n + i
    int *fcnt = nullptr, *scnt = nullptr, *fidx = nullptr, *sidx = nullptr;
    double *fw = nullptr, *sw = nullptr;
    double2 *fgw = nullptr, *sgw = nullptr;
    // cell sort of fluid and solid particles
    unsigned long long *fkeys = nullptr, *skeys = nullptr;
    int *fvals = nullptr, *svals = nullptr;
};

__host__ __device__ double kernel_w(double r, double h) {
    double const q = r / h;
    double const k = h * h * h * kPi;
    if (q <= 1.0) return (1.0 + q * q * (q * 0.75 - 1.5)) / k;
    if (q <= 2.0) {
        double const t = 2.0 - q;
        return ((t * t * t) / 4.0) / k;
    }
    return 0.0;
}

__host__ __device__ double kernel_dw(double r, double h) {
    double const q = r / h;
    double const k = h * h * h * kPi;
    if (q <= 1.0) return (-3.0 * r / (h * h) + 2.25 * r * r / (h * h * h)) / k;
    if (q <= 2.0) {
        double const t = 2.0 - q;
        return (-3.0 * t * t / (4.0 * h)) / k;
    }
    return 0.0;
}

__device__ unsigned long long cell_key(double2 p, double cell) {
    long long const gx = static_cast<long long>(floor(p.x / cell)) + (1ll << 30);
    long long const gy = static_cast<long long>(floor(p.y / cell)) + (1ll << 30);
    return (static_cast<unsigned long long>(gy) << 32) | static_cast<unsigned long long>(gx);
}

__global__ void k_keys(double2 const* x, size_t n, double cell, unsigned long long* keys, int* vals) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    keys[i] = cell_key(x[i], cell);
    vals[i] = int(i);
}

__device__ size_t lower_bound(unsigned long long const* keys, size_t n, unsigned long long key) {
    size_t lo = 0, hi = n;
    while (lo < hi) {
        size_t const mid = (lo + hi) / 2;
        if (keys[mid] < key) {
            lo = mid + 1;
        } else {
            hi = mid;
        }
    }
    return lo;
}

// Neighbours of fluid particle i among `other` (fluid or solid) within
// 2 * support, self excluded, ordered by (distance, index), at most kMax.
__global__ void k_neighbors(Sim s, double2 const* other, size_t n_other,
                            unsigned long long const* keys, int const* vals, bool self_set,
                            int* cnt, int* idx, double* w, double2* gw) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double const h = s.p.support;
    double const cell = 2.0 * h;
    double2 const xi = s.x[i];
    unsigned long long const k0 = cell_key(xi, cell);
    double ld[kMax];
    int lj[kMax];
    int m = 0;
    for (int dy = -1; dy <= 1; ++dy) {
        for (int dx = -1; dx <= 1; ++dx) {
            unsigned long long const key =
              k0 + (static_cast<unsigned long long>(static_cast<long long>(dy)) << 32) +
              static_cast<unsigned long long>(static_cast<long long>(dx));
            for (size_t q = lower_bound(keys, n_other, key); q < n_other && keys[q] == key; ++q) {
                int const j = vals[q];
                if (self_set && size_t(j) == i) continue;
                double const ddx = other[j].x - xi.x;
                double const ddy = other[j].y - xi.y;
                double const d = sqrt(ddx * ddx + ddy * ddy);
                if (!(d < cell)) continue;
                // sorted insertion on (d, j), keeping the first kMax
                int pos = m;
                while (pos > 0 && (ld[pos - 1] > d || (ld[pos - 1] == d && lj[pos - 1] > j))) --pos;
                if (pos >= kMax) continue;
                int const last = m < kMax ? m : kMax - 1;
                for (int t = last; t > pos; --t) {
                    ld[t] = ld[t - 1];
                    lj[t] = lj[t - 1];
                }
                ld[pos] = d;
                lj[pos] = j;
                if (m < kMax) ++m;
            }
        }
    }
    cnt[i] = m;
    for (int k = 0; k < m; ++k) {
        size_t const e = size_t(k) * s.n + i;
        int const j = lj[k];
        double const d = ld[k];
        idx[e] = j;
        w[e] = kernel_w(d, h);
        double2 g = make_double2(0.0, 0.0);
        if (d > 0.0) {
            double const dw = kernel_dw(d, h);
            g = make_double2((xi.x - other[j].x) / d * dw, (xi.y - other[j].y) / d * dw);
        }
        gw[e] = g;
    }
}

__device__ double q_of(double p, double rho) {
    double const d = rho * rho;
    return d != 0.0 ? p / d : 0.0;
}

__global__ void k_density_alpha(Sim s, int new_frame) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double const rho0 = s.p.rho0, fvol = s.p.fluid_volume;
    double const fmass = rho0 * fvol;
    double d = fvol * rho0 * kernel_w(0.0, s.p.support);
    double2 sum = make_double2(0.0, 0.0);
    double sdot = 0.0;
    int const cf = s.fcnt[i];
    for (int k = 0; k < cf; ++k) {
        size_t const e = size_t(k) * s.n + i;
        d += s.fw[e] * fmass;
        double2 const m = make_double2(fmass * s.fgw[e].x, fmass * s.fgw[e].y);
        sum.x += m.x;
        sum.y += m.y;
        sdot += m.x * m.x + m.y * m.y;
    }
    int const cs = s.scnt[i];
    double db = 0.0;
    for (int k = 0; k < cs; ++k) {
        size_t const e = size_t(k) * s.n + i;
        double const vs = s.vols[s.sidx[e]];
        db += s.sw[e] * (rho0 * vs);
        sum.x += vs * rho0 * s.sgw[e].x;
        sum.y += vs * rho0 * s.sgw[e].y;
    }
    d += db;
    s.rho[i] = d;
    double alpha = 0.0;
    if (cf + cs) {
        double const denom = sum.x * sum.x + sum.y * sum.y + sdot;
        alpha = denom != 0.0 ? d * d / denom : 0.0;
    }
    s.alpha[i] = alpha;
    if (new_frame) {
        s.kdiv[i] = 0.0;
        s.kdens[i] = 0.0;
    }
    s.qdiv[i] = q_of(s.kdiv[i], d);
    s.qdens[i] = q_of(s.kdens[i], d);
}

__global__ void k_apply(Sim s, double const* q, double dt, int external) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double const rho0 = s.p.rho0;
    double const neg_fmass = -(rho0 * s.p.fluid_volume);
    double2 v = s.v[i];
    if (external) {
        double const denom = rho0 * s.p.fluid_volume;
        v.y += dt * (-(s.p.mass * s.p.gravity)) / denom;
    }
    double const qi = q[i];
    double2 acc = make_double2(0.0, 0.0);
    int const c = s.fcnt[i];
    for (int k = 0; k < c; ++k) {
        size_t const e = size_t(k) * s.n + i;
        double const f = neg_fmass * (qi + q[s.fidx[e]]);
        acc.x += f * s.fgw[e].x;
        acc.y += f * s.fgw[e].y;
    }
    v.x += dt * acc.x;
    v.y += dt * acc.y;
    acc = make_double2(0.0, 0.0);
    int const cs = s.scnt[i];
    for (int k = 0; k < cs; ++k) {
        size_t const e = size_t(k) * s.n + i;
        double const f = -(rho0 * s.vols[s.sidx[e]]) * qi;
        acc.x += f * s.sgw[e].x;
        acc.y += f * s.sgw[e].y;
    }
    v.x += dt * acc.x;
    v.y += dt * acc.y;
    s.v[i] = v;
}

__device__ double divergence(Sim const& s, size_t i) {
    double const rho0 = s.p.rho0;
    double const fmass = rho0 * s.p.fluid_volume;
    double2 const vi = s.v[i];
    double d = 0.0;
    int const c = s.fcnt[i];
    for (int k = 0; k < c; ++k) {
        size_t const e = size_t(k) * s.n + i;
        double2 const vj = s.v[s.fidx[e]];
        d += fmass * ((vi.x - vj.x) * s.fgw[e].x + (vi.y - vj.y) * s.fgw[e].y);
    }
    double db = 0.0;
    int const cs = s.scnt[i];
    for (int k = 0; k < cs; ++k) {
        size_t const e = size_t(k) * s.n + i;
        int const j = s.sidx[e];
        db += (rho0 * s.vols[j]) * (vi.x * s.sgw[e].x + vi.y * s.sgw[e].y);  // solids at rest
    }
    return d + db;
}

// Divergence step (kind 0) or density step (kind 1) of one solver iteration.
__global__ void k_kappa(Sim s, double dt, int kind) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double const d = divergence(s, i);
    s.div[i] = d;
    if (kind == 0) {
        double const kappa = d > 0.0 ? d * s.alpha[i] / dt : 0.0;
        s.kdiv[i] = kappa;
        s.qdiv[i] = q_of(kappa, s.rho[i]);
    } else {
        double star = s.rho[i] + dt * d;
        if (star < 0.0) star = 0.0;
        s.rho_star[i] = star;
        double const delta = star - s.p.rho0;
        double const kappa = delta > 0.0 ? delta * s.alpha[i] / (dt * dt) : 0.0;
        s.kdens[i] = kappa;
        s.qdens[i] = q_of(kappa, s.rho[i]);
    }
}

// ---------------------------------------------------------------- IISPH

// External gravity and dii = -dt^2 sum_j m_j gradW_ij / rho_i^2 over fluid
// then boundary neighbours (iisph_ops.cpp:20-90); zero initial pressures.
__global__ void k_iisph_dii(Sim s, double dt) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double const rho0 = s.p.rho0;
    double const fmass = rho0 * s.p.fluid_volume;
    s.v[i].y += dt * (-(s.p.mass * s.p.gravity)) / fmass;
    double const denom = s.rho[i] * s.rho[i];
    double2 dii = make_double2(0.0, 0.0);
    int const cf = s.fcnt[i];
    if (cf && denom != 0.0) {
        double2 g = make_double2(0.0, 0.0);
        for (int k = 0; k < cf; ++k) {
            size_t const e = size_t(k) * s.n + i;
            g.x += fmass * s.fgw[e].x;
            g.y += fmass * s.fgw[e].y;
        }
        dii = make_double2(-dt * dt * g.x / denom, -dt * dt * g.y / denom);
    }
    int const cs = s.scnt[i];
    if (cs && denom != 0.0) {
        double2 g = make_double2(0.0, 0.0);
        for (int k = 0; k < cs; ++k) {
            size_t const e = size_t(k) * s.n + i;
            double const m = rho0 * s.vols[s.sidx[e]];
            g.x += m * s.sgw[e].x;
            g.y += m * s.sgw[e].y;
        }
        dii.x += -dt * dt * g.x / denom;
        dii.y += -dt * dt * g.y / denom;
    }
    s.dii[i] = dii;
    s.pres[i] = 0.0;
}

// aii and the predicted density rho* (iisph_ops.cpp:92-200); the boundary
// is at rest.
__global__ void k_iisph_aii(Sim s, double dt) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double const rho0 = s.p.rho0;
    double const fmass = rho0 * s.p.fluid_volume;
    double2 const dii = s.dii[i];
    double2 const vi = s.v[i];
    double aii = 0.0, dd = 0.0;
    int const cf = s.fcnt[i];
    for (int k = 0; k < cf; ++k) {
        size_t const e = size_t(k) * s.n + i;
        int const j = s.fidx[e];
        double2 const g = s.fgw[e];
        double const dj = s.rho[j] * s.rho[j];
        if (dj != 0.0) {
            // dji = -dij = dt^2 m gradW_ij / rho_j^2
            double2 const dji = make_double2(dt * dt * fmass * g.x / dj, dt * dt * fmass * g.y / dj);
            aii += fmass * ((dii.x - dji.x) * g.x + (dii.y - dji.y) * g.y);
        }
        dd += dt * fmass * ((vi.x - s.v[j].x) * g.x + (vi.y - s.v[j].y) * g.y);
    }
    int const cs = s.scnt[i];
    for (int k = 0; k < cs; ++k) {
        size_t const e = size_t(k) * s.n + i;
        double const m = s.vols[s.sidx[e]] * rho0;
        double2 const g = s.sgw[e];
        aii += m * (dii.x * g.x + dii.y * g.y);
        dd += dt * m * (vi.x * g.x + vi.y * g.y);
    }
    s.aii[i] = aii;
    s.rho_star[i] = s.rho[i] + dd;
}

// sum_j dij pj over fluid neighbours (iisph_ops.cpp:202-235).
__global__ void k_iisph_sdp(Sim s, double dt) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double const fmass = s.p.rho0 * s.p.fluid_volume;
    double2 sum = make_double2(0.0, 0.0);
    int const cf = s.fcnt[i];
    for (int k = 0; k < cf; ++k) {
        size_t const e = size_t(k) * s.n + i;
        int const j = s.fidx[e];
        double const dj = s.rho[j] * s.rho[j];
        if (dj == 0.0) continue;
        double const c = -dt * dt * fmass * s.pres[j] / dj;
        sum.x += c * s.fgw[e].x;
        sum.y += c * s.fgw[e].y;
    }
    s.sdp[i] = sum;
}

// beta_i (iisph_ops.cpp:237-330) and the relaxed Jacobi pressure update
// p_i <- max(0, mix(p_i, (rho0 - rho*_i - beta_i) / aii, omega))
// (iisph_ops.cpp:332-425).
__global__ void k_iisph_pressures(Sim s, double dt, double omega) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double const rho0 = s.p.rho0;
    double const fmass = rho0 * s.p.fluid_volume;
    double const pi = s.pres[i];
    double2 const si = s.sdp[i];
    double beta = 0.0;
    int const cf = s.fcnt[i];
    for (int k = 0; k < cf; ++k) {
        size_t const e = size_t(k) * s.n + i;
        int const j = s.fidx[e];
        double2 const g = s.fgw[e];
        double const dj = s.rho[j] * s.rho[j];
        double2 dji = make_double2(0.0, 0.0);
        if (dj != 0.0) dji = make_double2(dt * dt * fmass * g.x / dj, dt * dt * fmass * g.y / dj);
        double const pj = s.pres[j];
        double2 const djj = s.dii[j];
        double2 const sj = s.sdp[j];
        double const tx = si.x - djj.x * pj - (sj.x - dji.x * pi);
        double const ty = si.y - djj.y * pj - (sj.y - dji.y * pi);
        beta += fmass * (tx * g.x + ty * g.y);
    }
    int const cs = s.scnt[i];
    for (int k = 0; k < cs; ++k) {
        size_t const e = size_t(k) * s.n + i;
        beta += rho0 * s.vols[s.sidx[e]] * (si.x * s.sgw[e].x + si.y * s.sgw[e].y);
    }
    double const alpha = s.aii[i];
    double out = pi;
    if (alpha != 0.0) {
        double const p_new = (rho0 - s.rho_star[i] - beta) / alpha;
        out = pi * (1.0 - omega) + p_new * omega;
        if (out < 0.0) out = 0.0;
    }
    s.pres_next[i] = out;
}

// q_i = p_i / rho_i^2 of the final pressures, for apply_pressures_in_place.
__global__ void k_iisph_q(Sim s) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    s.qdens[i] = q_of(s.pres[i], s.rho[i]);
}

__global__ void k_positions(Sim s, double dt) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    s.x[i].x += dt * s.v[i].x;
    s.x[i].y += dt * s.v[i].y;
}

// ------------------------------------------------------- IISPH_AP / PSEUDO_AP

// integrate_velocities_in_place with the gravity force (dynamics.cpp:24-37).
__global__ void k_external(Sim s, double dt) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double const denom = s.p.rho0 * s.p.fluid_volume;
    s.v[i].y += dt * (-(s.p.mass * s.p.gravity)) / denom;
}

// iisph_ap_density_stars_and_diagonals (iisph_ap_ops.cpp:19-90) and its
// pseudo form (iisph_pseudo_ap_ops.cpp:19-117, without the dt^2): diagonal
// -dt^2 (|sum m gradW|^2 + m_i sum_f m |gradW|^2) / rho^2 and
// rho* = rho + dt * divergence; the boundary is at rest.
__global__ void k_ap_diag(Sim s, double dt, int pseudo) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double const rho0 = s.p.rho0;
    double const fmass = rho0 * s.p.fluid_volume;
    int const cf = s.fcnt[i];
    int const cs = s.scnt[i];
    double const rho = s.rho[i];
    if (!(cf + cs)) {
        s.rho_star[i] = rho;
        s.aii[i] = 0.0;
        return;
    }
    double2 const vi = s.v[i];
    double2 sum = make_double2(0.0, 0.0);
    double sdot = 0.0, div = 0.0;
    for (int k = 0; k < cf; ++k) {
        size_t const e = size_t(k) * s.n + i;
        double2 const g = s.fgw[e];
        double2 const vj = s.v[s.fidx[e]];
        sum.x += fmass * g.x;
        sum.y += fmass * g.y;
        sdot += fmass * (g.x * g.x + g.y * g.y);
        div += fmass * ((vi.x - vj.x) * g.x + (vi.y - vj.y) * g.y);
    }
    for (int k = 0; k < cs; ++k) {
        size_t const e = size_t(k) * s.n + i;
        double2 const g = s.sgw[e];
        double const m = s.vols[s.sidx[e]] * rho0;
        sum.x += m * g.x;
        sum.y += m * g.y;
        div += m * (vi.x * g.x + vi.y * g.y);
    }
    double const denom = rho * rho;
    double numer = -(sum.x * sum.x + sum.y * sum.y + fmass * sdot);
    if (!pseudo) numer *= dt * dt;
    s.aii[i] = denom != 0.0 ? numer / denom : 0.0;
    s.rho_star[i] = rho + dt * div;
}

// compute_pressure_accelerations (pressure.cpp:83-178) of the current
// pressures; under PSEUDO_AP the same sum gives the displacements
// (iisph_pseudo_ap_ops.cpp:119-224).
__global__ void k_ap_accel(Sim s) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double const rho0 = s.p.rho0;
    double const fmass = rho0 * s.p.fluid_volume;
    double const qi = q_of(s.pres[i], s.rho[i]);
    double2 a = make_double2(0.0, 0.0);
    int const cf = s.fcnt[i];
    for (int k = 0; k < cf; ++k) {
        size_t const e = size_t(k) * s.n + i;
        int const j = s.fidx[e];
        double const f = -fmass * (qi + q_of(s.pres[j], s.rho[j]));
        a.x += f * s.fgw[e].x;
        a.y += f * s.fgw[e].y;
    }
    int const cs = s.scnt[i];
    for (int k = 0; k < cs; ++k) {
        size_t const e = size_t(k) * s.n + i;
        double const f = -(rho0 * s.vols[s.sidx[e]]) * qi;
        a.x += f * s.sgw[e].x;
        a.y += f * s.sgw[e].y;
    }
    s.acc[i] = a;
}

// One relaxed Jacobi step p <- max(0, p + omega (s - A p) / diag)
// (iisph_ap_ops.cpp:92-194, iisph_pseudo_ap_ops.cpp:226-323).
__global__ void k_ap_iterate(Sim s, double dt, double omega, int pseudo) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double const rho0 = s.p.rho0;
    double const fmass = rho0 * s.p.fluid_volume;
    int const cf = s.fcnt[i];
    int const cs = s.scnt[i];
    double const diag = s.aii[i];
    if ((!cf && !cs) || (pseudo && diag == 0.0)) {
        s.pres[i] = 0.0;
        return;
    }
    double2 const ai = s.acc[i];
    double api = 0.0;
    for (int k = 0; k < cf; ++k) {
        size_t const e = size_t(k) * s.n + i;
        double2 const aj = s.acc[s.fidx[e]];
        api += fmass * ((ai.x - aj.x) * s.fgw[e].x + (ai.y - aj.y) * s.fgw[e].y);
    }
    for (int k = 0; k < cs; ++k) {
        size_t const e = size_t(k) * s.n + i;
        api += (rho0 * s.vols[s.sidx[e]]) * (ai.x * s.sgw[e].x + ai.y * s.sgw[e].y);
    }
    if (!pseudo) api *= dt * dt;
    double const source = rho0 - s.rho_star[i];
    double p = s.pres[i] + (diag != 0.0 ? omega * (source - api) / diag : 0.0);
    s.pres[i] = p < 0.0 ? 0.0 : p;
}

// integrate_velocities_and_positions_in_place (dynamics.cpp:53-63), or the
// PSEUDO_AP update x += dt v* + dx, v = v* + dx / dt
// (iisph_pseudo_ap_ops.cpp:325-343).
__global__ void k_ap_finish(Sim s, double dt, int pseudo) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double2 const a = s.acc[i];
    double2 v = s.v[i];
    double2 x = s.x[i];
    if (!pseudo) {
        v.x += dt * a.x;
        v.y += dt * a.y;
        x.x += dt * v.x;
        x.y += dt * v.y;
    } else {
        x.x += dt * v.x + a.x;
        x.y += dt * v.y + a.y;
        if (dt != 0.0) {
            v.x += a.x / dt;
            v.y += a.y / dt;
        }
    }
    s.v[i] = v;
    s.x[i] = x;
}

// ---------------------------------------------------------------- PCISPH

// Velocity after the external force, v_ext = v + (dt / m) F_gravity
// (pcisph.cpp:36-80), and zero pressures.
__global__ void k_pc_init(Sim s, double dt) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double const m = s.p.mass;
    double2 v = s.v[i];
    v.y += (dt / m) * (-(m * s.p.gravity));
    s.vext[i] = v;
    s.pres[i] = 0.0;
    s.fpres[i] = make_double2(0.0, 0.0);
}

// Predicted velocity and position of one pass (pcisph.cpp:82-110).
__global__ void k_pc_predict(Sim s, double dt, int pass) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double const mult = dt / s.p.mass;
    double2 v = s.vext[i];
    if (pass > 0) {
        v.x += mult * s.fpres[i].x;
        v.y += mult * s.fpres[i].y;
    }
    s.vstar[i] = v;
    s.xstar[i] = make_double2(s.x[i].x + dt * v.x, s.x[i].y + dt * v.y);
}

// The fixed lists' kernels at the predicted positions
// (compute_neighbor_distances_and_vectors_to, neighborhood.cpp:154-176, then
// the kernels of neighborhood.cpp:178-210).
__global__ void k_pc_kernels(Sim s) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double const h = s.p.support;
    double2 const xi = s.xstar[i];
    for (int set = 0; set < 2; ++set) {
        int const c = set ? s.scnt[i] : s.fcnt[i];
        int const* idx = set ? s.sidx : s.fidx;
        double2 const* other = set ? s.xs : s.xstar;
        double* w = set ? s.sw : s.fw;
        double2* gw = set ? s.sgw : s.fgw;
        for (int k = 0; k < c; ++k) {
            size_t const e = size_t(k) * s.n + i;
            double2 const xj = other[idx[e]];
            double const vx = xj.x - xi.x, vy = xj.y - xi.y;
            double const d = sqrt(vx * vx + vy * vy);
            w[e] = kernel_w(d, h);
            double2 g = make_double2(0.0, 0.0);
            if (d > 0.0) {
                double const dw = kernel_dw(d, h);
                g = make_double2(-vx / d * dw, -vy / d * dw);
            }
            gw[e] = g;
        }
    }
}

// pcisph_compute_densities, pcisph_accumulate_density_from_solids and
// pcisph_update_pressures (pcisph_ops.cpp:18-76).
__global__ void k_pc_density(Sim s, double denom) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double const m = s.p.mass;
    double const rho0 = s.p.rho0;
    double ws = kernel_w(0.0, s.p.support);
    int const cf = s.fcnt[i];
    for (int k = 0; k < cf; ++k) ws += s.fw[size_t(k) * s.n + i];
    double rho = m * ws;
    int const cs = s.scnt[i];
    if (cs) {
        double vf = 0.0;
        for (int k = 0; k < cs; ++k) {
            size_t const e = size_t(k) * s.n + i;
            vf += s.vols[s.sidx[e]] * s.sw[e];
        }
        rho += rho0 * vf;
    }
    s.rho[i] = rho;
    double const err = rho - rho0;
    s.pres[i] += (err > 0.0 ? err : 0.0) / denom;
}

// pcisph_accumulate_pressure_forces with the artificial viscosity
// (alpha = viscosity, beta = 2, N2 = 0.01 h^2) and
// pcisph_accumulate_pressure_forces_from_solids (pcisph_ops.cpp:78-178).
__global__ void k_pc_forces(Sim s, double viscosity) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double const m = s.p.mass;
    double const rho0 = s.p.rho0;
    double const H = s.p.support;
    double const N2 = 0.01 * H * H;
    double const rho = s.rho[i];
    double const pors = s.pres[i] / (rho * rho);
    double2 f = make_double2(0.0, 0.0);
    int const cf = s.fcnt[i];
    if (cf) {
        double2 const xi = s.xstar[i];
        double2 const vi = s.vstar[i];
        double2 pf = make_double2(0.0, 0.0);
        for (int k = 0; k < cf; ++k) {
            size_t const e = size_t(k) * s.n + i;
            int const j = s.fidx[e];
            double2 const g = s.fgw[e];
            double const rj = s.rho[j];
            double const c = pors + s.pres[j] / (rj * rj);
            pf.x += c * g.x;
            pf.y += c * g.y;
            double const tx = s.xstar[j].x - xi.x, ty = s.xstar[j].y - xi.y;
            double const dvr = tx * (s.vstar[j].x - vi.x) + ty * (s.vstar[j].y - vi.y);
            if (dvr < 0.0) {
                double const dist = sqrt(tx * tx + ty * ty);
                double const mu = H * dvr / (dist + N2);
                double const den = (rho + rj) / 2.0;
                double const visc = ((-1.0 * viscosity * mu) + (2.0 * mu * mu)) / den;
                pf.x += visc * g.x;
                pf.y += visc * g.y;
            }
        }
        f.x += -(m * m) * pf.x;
        f.y += -(m * m) * pf.y;
    }
    int const cs = s.scnt[i];
    if (cs) {
        double2 vg = make_double2(0.0, 0.0);
        for (int k = 0; k < cs; ++k) {
            size_t const e = size_t(k) * s.n + i;
            double const vol = s.vols[s.sidx[e]];
            vg.x += vol * s.sgw[e].x;
            vg.y += vol * s.sgw[e].y;
        }
        f.x += -m * rho0 * pors * vg.x;
        f.y += -m * rho0 * pors * vg.y;
    }
    s.fpres[i] = f;
}

// v = v_ext + (dt / m) F_pressure, x += dt v (pcisph.cpp:150-164).
__global__ void k_pc_final(Sim s, double dt) {
    size_t const i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= s.n) return;
    double const mult = dt / s.p.mass;
    double2 v = s.vext[i];
    v.x += mult * s.fpres[i].x;
    v.y += mult * s.fpres[i].y;
    s.v[i] = v;
    s.x[i].x += dt * v.x;
    s.x[i].y += dt * v.y;
}

template <class T>
T* dalloc(size_t count) {
    void* p = nullptr;
    if (cudaMalloc(&p, count * sizeof(T) + 16) != cudaSuccess) return nullptr;
    return static_cast<T*>(p);
}

unsigned grid(size_t n) { return unsigned((n + 127) / 128); }

void sort_cells(double2 const* x, size_t n, double cell, unsigned long long* keys, int* vals) {
    if (!n) return;
    k_keys<<<grid(n), 128>>>(x, n, cell, keys, vals);
    thrust::sort_by_key(thrust::device_ptr<unsigned long long>(keys),
                        thrust::device_ptr<unsigned long long>(keys + n),
                        thrust::device_ptr<int>(vals));
}

}  // namespace

extern "C" {

typedef struct fp64_params {
    double support, rho0, mass, fluid_volume, gravity;
} fp64_params;

int fp64_destroy(void* h);

int fp64_create(fp64_params const* p, double const* solid_xy, double const* solid_vols, size_t ns,
                double const* fluid_xy, double const* fluid_v, size_t n, void** out) {
    Sim* s = new Sim;
    s->p = Params{p->support, p->rho0, p->mass, p->fluid_volume, p->gravity};
    s->n = n;
    s->ns = ns;
    size_t const E = n * kMax;
    s->x = dalloc<double2>(n);
    s->v = dalloc<double2>(n);
    s->xs = dalloc<double2>(ns);
    s->vols = dalloc<double>(ns);
    s->rho = dalloc<double>(n);
    s->alpha = dalloc<double>(n);
    s->kdiv = dalloc<double>(n);
    s->kdens = dalloc<double>(n);
    s->qdiv = dalloc<double>(n);
    s->qdens = dalloc<double>(n);
    s->rho_star = dalloc<double>(n);
    s->div = dalloc<double>(n);
    s->dii = dalloc<double2>(n);
    s->sdp = dalloc<double2>(n);
    s->aii = dalloc<double>(n);
    s->pres = dalloc<double>(n);
    s->pres_next = dalloc<double>(n);
    s->vext = dalloc<double2>(n);
    s->vstar = dalloc<double2>(n);
    s->xstar = dalloc<double2>(n);
    s->fpres = dalloc<double2>(n);
    s->acc = dalloc<double2>(n);
    s->fcnt = dalloc<int>(n);
    s->scnt = dalloc<int>(n);
    s->fidx = dalloc<int>(E);
    s->sidx = dalloc<int>(E);
    s->fw = dalloc<double>(E);
    s->sw = dalloc<double>(E);
    s->fgw = dalloc<double2>(E);
    s->sgw = dalloc<double2>(E);
    s->fkeys = dalloc<unsigned long long>(n);
    s->skeys = dalloc<unsigned long long>(ns);
    s->fvals = dalloc<int>(n);
    s->svals = dalloc<int>(ns);
    if (!s->sgw || !s->svals || !s->fvals || !s->dii || !s->sdp || !s->aii || !s->pres ||
        !s->pres_next || !s->vext || !s->vstar || !s->xstar || !s->fpres || !s->acc) {
        fp64_destroy(s);
        return 12;
    }
    cudaMemcpy(s->x, fluid_xy, 16 * n, cudaMemcpyHostToDevice);
    if (fluid_v) {
        cudaMemcpy(s->v, fluid_v, 16 * n, cudaMemcpyHostToDevice);
    } else {
        cudaMemset(s->v, 0, 16 * n);
    }
    cudaMemcpy(s->xs, solid_xy, 16 * ns, cudaMemcpyHostToDevice);
    cudaMemcpy(s->vols, solid_vols, 8 * ns, cudaMemcpyHostToDevice);
    cudaMemset(s->kdiv, 0, 8 * n);
    cudaMemset(s->kdens, 0, 8 * n);
    sort_cells(s->xs, ns, 2.0 * s->p.support, s->skeys, s->svals);
    *out = s;
    return cudaGetLastError() == cudaSuccess ? 0 : 1000;
}

int fp64_destroy(void* h) {
    Sim* s = static_cast<Sim*>(h);
    void* ptrs[] = {s->x,    s->v,    s->xs,    s->vols,  s->rho,   s->alpha, s->kdiv,
                    s->kdens, s->qdiv, s->qdens, s->rho_star, s->div, s->fcnt,  s->scnt,
                    s->fidx, s->sidx, s->fw,    s->sw,    s->fgw,   s->sgw,   s->fkeys,
                    s->skeys, s->fvals, s->svals, s->dii, s->sdp, s->aii, s->pres,
                    s->pres_next, s->vext, s->vstar, s->xstar, s->fpres, s->acc};
    for (void* p : ptrs) cudaFree(p);
    delete s;
    return 0;
}

// One DFSPH_P sub-step of length dt with the given iteration counts.
int fp64_sub_step(void* h, double dt, int new_frame, int div_iters, int dens_iters) {
    Sim& s = *static_cast<Sim*>(h);
    size_t const n = s.n;
    double const cell = 2.0 * s.p.support;
    sort_cells(s.x, n, cell, s.fkeys, s.fvals);
    k_neighbors<<<grid(n), 128>>>(s, s.x, n, s.fkeys, s.fvals, true, s.fcnt, s.fidx, s.fw, s.fgw);
    k_neighbors<<<grid(n), 128>>>(s, s.xs, s.ns, s.skeys, s.svals, false, s.scnt, s.sidx, s.sw,
                                  s.sgw);
    k_density_alpha<<<grid(n), 128>>>(s, new_frame);
    k_apply<<<grid(n), 128>>>(s, s.qdiv, dt, 0);
    for (int it = 0; it < div_iters; ++it) {
        k_kappa<<<grid(n), 128>>>(s, dt, 0);
        k_apply<<<grid(n), 128>>>(s, s.qdiv, dt, 0);
    }
    k_apply<<<grid(n), 128>>>(s, s.qdens, dt, 1);
    for (int it = 0; it < dens_iters; ++it) {
        k_kappa<<<grid(n), 128>>>(s, dt, 1);
        k_apply<<<grid(n), 128>>>(s, s.qdens, dt, 0);
    }
    k_positions<<<grid(n), 128>>>(s, dt);
    cudaError_t const e = cudaDeviceSynchronize();
    return e == cudaSuccess ? 0 : 1000;
}

// One IISPH sub-step of length dt running `iters` pressure iterations with
// relaxation omega (the sub-step of emerald/sph2d_box/iisph.cpp:23-151).
int fp64_sub_step_iisph(void* h, double dt, int iters, double omega) {
    Sim& s = *static_cast<Sim*>(h);
    size_t const n = s.n;
    double const cell = 2.0 * s.p.support;
    sort_cells(s.x, n, cell, s.fkeys, s.fvals);
    k_neighbors<<<grid(n), 128>>>(s, s.x, n, s.fkeys, s.fvals, true, s.fcnt, s.fidx, s.fw, s.fgw);
    k_neighbors<<<grid(n), 128>>>(s, s.xs, s.ns, s.skeys, s.svals, false, s.scnt, s.sidx, s.sw,
                                  s.sgw);
    k_density_alpha<<<grid(n), 128>>>(s, 0);
    k_iisph_dii<<<grid(n), 128>>>(s, dt);
    k_iisph_aii<<<grid(n), 128>>>(s, dt);
    for (int it = 0; it < iters; ++it) {
        k_iisph_sdp<<<grid(n), 128>>>(s, dt);
        k_iisph_pressures<<<grid(n), 128>>>(s, dt, omega);
        double* t = s.pres;
        s.pres = s.pres_next;
        s.pres_next = t;
    }
    k_iisph_q<<<grid(n), 128>>>(s);
    k_apply<<<grid(n), 128>>>(s, s.qdens, dt, 0);
    k_positions<<<grid(n), 128>>>(s, dt);
    cudaError_t const e = cudaDeviceSynchronize();
    return e == cudaSuccess ? 0 : 1000;
}

// One IISPH_AP (pseudo 0) or IISPH_PSEUDO_AP (pseudo 1) sub-step of length dt
// running `iters` Jacobi iterations with relaxation omega.
int fp64_sub_step_ap(void* h, double dt, int iters, double omega, int pseudo) {
    Sim& s = *static_cast<Sim*>(h);
    size_t const n = s.n;
    double const cell = 2.0 * s.p.support;
    sort_cells(s.x, n, cell, s.fkeys, s.fvals);
    k_neighbors<<<grid(n), 128>>>(s, s.x, n, s.fkeys, s.fvals, true, s.fcnt, s.fidx, s.fw, s.fgw);
    k_neighbors<<<grid(n), 128>>>(s, s.xs, s.ns, s.skeys, s.svals, false, s.scnt, s.sidx, s.sw,
                                  s.sgw);
    k_density_alpha<<<grid(n), 128>>>(s, 0);
    k_external<<<grid(n), 128>>>(s, dt);
    k_ap_diag<<<grid(n), 128>>>(s, dt, pseudo);
    cudaMemset(s.pres, 0, 8 * n);
    for (int it = 0; it < iters; ++it) {
        k_ap_accel<<<grid(n), 128>>>(s);
        k_ap_iterate<<<grid(n), 128>>>(s, dt, omega, pseudo);
    }
    k_ap_accel<<<grid(n), 128>>>(s);
    k_ap_finish<<<grid(n), 128>>>(s, dt, pseudo);
    cudaError_t const e = cudaDeviceSynchronize();
    return e == cudaSuccess ? 0 : 1000;
}

// One PCISPH sub-step of length dt running `passes` predictor-corrector
// passes, with the PCISPH viscosity and the pressure-correction denominator
// of Simulation_config.
int fp64_sub_step_pcisph(void* h, double dt, int passes, double viscosity, double denom) {
    Sim& s = *static_cast<Sim*>(h);
    size_t const n = s.n;
    double const cell = 2.0 * s.p.support;
    sort_cells(s.x, n, cell, s.fkeys, s.fvals);
    k_neighbors<<<grid(n), 128>>>(s, s.x, n, s.fkeys, s.fvals, true, s.fcnt, s.fidx, s.fw, s.fgw);
    k_neighbors<<<grid(n), 128>>>(s, s.xs, s.ns, s.skeys, s.svals, false, s.scnt, s.sidx, s.sw,
                                  s.sgw);
    k_pc_init<<<grid(n), 128>>>(s, dt);
    for (int pass = 0; pass < passes; ++pass) {
        k_pc_predict<<<grid(n), 128>>>(s, dt, pass);
        k_pc_kernels<<<grid(n), 128>>>(s);
        k_pc_density<<<grid(n), 128>>>(s, denom);
        k_pc_forces<<<grid(n), 128>>>(s, viscosity);
    }
    k_pc_final<<<grid(n), 128>>>(s, dt);
    cudaError_t const e = cudaDeviceSynchronize();
    return e == cudaSuccess ? 0 : 1000;
}

// "x", "v" (2 doubles per particle), "densities", "alphas", "pressures"
// (IISPH), "counts".
int fp64_get(void* h, char const* name, double* out) {
    Sim& s = *static_cast<Sim*>(h);
    size_t const n = s.n;
    if (!std::strcmp(name, "x")) return cudaMemcpy(out, s.x, 16 * n, cudaMemcpyDeviceToHost) ? 1000 : 0;
    if (!std::strcmp(name, "v")) return cudaMemcpy(out, s.v, 16 * n, cudaMemcpyDeviceToHost) ? 1000 : 0;
    if (!std::strcmp(name, "densities")) {
        return cudaMemcpy(out, s.rho, 8 * n, cudaMemcpyDeviceToHost) ? 1000 : 0;
    }
    if (!std::strcmp(name, "pressures")) {
        return cudaMemcpy(out, s.pres, 8 * n, cudaMemcpyDeviceToHost) ? 1000 : 0;
    }
    if (!std::strcmp(name, "alphas")) {
        return cudaMemcpy(out, s.alpha, 8 * n, cudaMemcpyDeviceToHost) ? 1000 : 0;
    }
    if (!std::strcmp(name, "counts")) {
        std::vector<int> c(n);
        if (cudaMemcpy(c.data(), s.fcnt, 4 * n, cudaMemcpyDeviceToHost)) return 1000;
        for (size_t i = 0; i < n; ++i) out[i] = c[i];
        return 0;
    }
    return 22;
}

}  // extern "C"
