// kernels.cu — CUDA kernels of the explicit time step (sm_100a).
//
// Data layout and roofline notes:
//  * The element kernel streams each honeycomb element's static record
//    (37 x 16 B planes: connectivity, dN/dX, hourglass base vectors, the
//    symmetric 12x12 hourglass stiffness, volume/material) and its state
//    (7 planes, read + written), gathers its 8 nodes' f64 position and
//    displacement through L2, and writes 24 f32 corner forces. All loads of
//    per-element data are 128-bit and coalesced (one plane = 512 B per warp).
//  * Force assembly is a gather, not an atomic scatter: each node sums its
//    incident (element, corner) forces in increasing element order over a
//    CSR built at set-up, in f64 — the order and precision of the reference's
//    serial scatter (src/kernel_simd.rs:573-586), so results are reproducible
//    run to run and identical to the reference's summation.
//  * Nothing here waits on another block or another GPU; every kernel is a
//    plain data-parallel pass whose only cross-block interaction is an
//    atomic integer count or an atomicMin on a bit pattern.
#include <cmath>
#include <cfloat>
#include <climits>
#include <math_constants.h>

#include <cub/cub.cuh>

#include "element.cuh"
#include "kernels.cuh"
#include "hencky.cuh"

namespace crush {

namespace {

constexpr int TPB = 256;
constexpr int FACE_TPB = 64;  // small blocks for the face pass: a few thousand latency-bound faces spread over more SMs

__host__ __device__ inline long long blocks_for(long long n, int tpb) { return (n + tpb - 1) / tpb; }

// Active-chunk iteration: thread g of the grid-stride loop handles entity
// active_entity(g) (mult threads per entity, lane = the thread's rank among
// them). Chunks are multiples of a warp, so the 32 lanes of a warp always
// take the same number of iterations and stay converged.
__device__ __forceinline__ long long active_total(const Active& a, long long n, int mult) {
    const long long chunks = a.list ? (long long)*a.count : (n + CHUNK - 1) / CHUNK;
    return chunks * CHUNK * mult;
}
__device__ __forceinline__ long long active_entity(const Active& a, long long g, int mult, int* lane) {
    const long long per = (long long)CHUNK * mult;
    const long long item = g / per, within = g - item * per;
    const long long chunk = a.list ? (long long)a.list[item] : item;
    *lane = (int)(within % mult);
    return chunk * CHUNK + within / mult;
}
#define FOR_ACTIVE(a, n, mult, g) \
    for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x, g##_end = active_total(a, n, mult); g < g##_end; \
         g += (long long)gridDim.x * blockDim.x)

// Grid of a FOR_ACTIVE launch: every chunk once, at most `cap` blocks.
inline unsigned active_grid(long long n, int mult, int tpb, long long cap) {
    const long long need = blocks_for(((n + CHUNK - 1) / CHUNK) * CHUNK * mult, tpb);
    return (unsigned)(need < 1 ? 1 : (need < cap ? need : cap));
}
constexpr long long GRID_CAP = 148 * 64;

// ---------------------------------------------------------------------------
// Set-up geometry (f64), restating src/element.rs:141-162 (HexGeometry::new)
// with the hourglass stiffness reduced directly to its rank-12 form.
// ---------------------------------------------------------------------------
__constant__ double c_xi[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                  {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
__constant__ double c_modes[4][8] = {{1, 1, -1, -1, -1, -1, 1, 1},
                                     {1, -1, -1, 1, -1, 1, 1, -1},
                                     {1, -1, 1, -1, 1, -1, 1, -1},
                                     {-1, 1, -1, 1, 1, -1, 1, -1}};

__device__ void shape_derivatives(double xi, double eta, double zeta, double dn[8][3]) {
    for (int i = 0; i < 8; ++i) {
        const double s0 = c_xi[i][0], s1 = c_xi[i][1], s2 = c_xi[i][2];
        dn[i][0] = 0.125 * s0 * (1.0 + s1 * eta) * (1.0 + s2 * zeta);
        dn[i][1] = 0.125 * s1 * (1.0 + s0 * xi) * (1.0 + s2 * zeta);
        dn[i][2] = 0.125 * s2 * (1.0 + s0 * xi) * (1.0 + s1 * eta);
    }
}

// First-row cofactor determinant and inverse of a row-major 3x3.
__device__ double det3d(const double* a) {
    double m11 = a[4] * a[8] - a[7] * a[5];
    double m12 = a[3] * a[8] - a[6] * a[5];
    double m13 = a[3] * a[7] - a[6] * a[4];
    return a[0] * m11 - a[1] * m12 + a[2] * m13;
}
__device__ bool inv3d(const double* a, double* r) {
    double m11 = a[4] * a[8] - a[7] * a[5];
    double m12 = a[3] * a[8] - a[6] * a[5];
    double m13 = a[3] * a[7] - a[6] * a[4];
    double det = a[0] * m11 - a[1] * m12 + a[2] * m13;
    if (det == 0.0) return false;
    r[0] = m11 / det;
    r[1] = -(a[1] * a[8] - a[7] * a[2]) / det;
    r[2] = (a[1] * a[5] - a[4] * a[2]) / det;
    r[3] = -m12 / det;
    r[4] = (a[0] * a[8] - a[6] * a[2]) / det;
    r[5] = -(a[0] * a[5] - a[3] * a[2]) / det;
    r[6] = m13 / det;
    r[7] = -(a[0] * a[7] - a[6] * a[1]) / det;
    r[8] = (a[0] * a[4] - a[3] * a[1]) / det;
    return true;
}

// J = dNᵀ x, grad = dN J⁻ᵀ (src/element.rs:43).
__device__ bool reference_gradients(const double x[8][3], const double dn[8][3], double g[8][3], double* det) {
    double j[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double s = dn[0][r] * x[0][c];
            for (int k = 1; k < 8; ++k) s = s + dn[k][r] * x[k][c];
            j[3 * r + c] = s;
        }
    double ji[9];
    if (!inv3d(j, ji)) return false;
    for (int i = 0; i < 8; ++i)
        for (int c = 0; c < 3; ++c) {
            double s = dn[i][0] * ji[3 * c];
            s = s + dn[i][1] * ji[3 * c + 1];
            s = s + dn[i][2] * ji[3 * c + 2];
            g[i][c] = s;
        }
    *det = det3d(j);
    return true;
}

// Element set-up (HexGeometry::new, src/element.rs:141-162): centre
// gradients, hourglass base vectors Γ, volume, consistent-mass row sums and
// the hourglass stiffness H = A G K Gᵀ A (A = (ΓᵀΓ)⁻¹), with G K Gᵀ
// accumulated per Gauss point as Mᵀ C M (M = (B_gp - B_c) Gᵀ, 6 x 12).
// Eight lanes per element, one per Gauss point: each lane evaluates its
// point's terms (the Mᵀ C M entries times det J, the consistent-mass
// entries, det J) and every sum over the points is taken in point order by
// shuffles, as a serial loop over the points adds them; the Gauss-Jordan
// inverse is repeated by every lane, and the H entries and the stores are
// split over the lanes. (One thread per element would keep the 12x12 and
// 8x8 sums in local memory.)
constexpr int GEO_LANES = 8, GEO_TPB = 128, GEO_PER_BLOCK = GEO_TPB / GEO_LANES;
__global__ void __launch_bounds__(GEO_TPB) k_setup_geometry8(long long e_begin, long long n_all, const double* __restrict__ pos,
                                                             const uint32_t* __restrict__ conn, const int32_t* __restrict__ part,
                                                             const double* __restrict__ mat, const int64_t* __restrict__ hc_index,
                                                             const uint32_t* __restrict__ elem_slot, long long stride,
                                                             float4* __restrict__ planes, double* __restrict__ volume_out,
                                                             double* __restrict__ lumped_out, double* __restrict__ dt_factor,
                                                             double* __restrict__ elem_mass, int* __restrict__ bad,
                                                             const int64_t* __restrict__ sc_index, long long n_sc,
                                                             double* __restrict__ sc_geo) {
    __shared__ double s_gkg[GEO_PER_BLOCK][78];
    __shared__ double s_h[GEO_PER_BLOCK][80];
    const int q = threadIdx.x % GEO_LANES, grp = threadIdx.x / GEO_LANES;
    const long long e_raw = e_begin + (long long)blockIdx.x * GEO_PER_BLOCK + grp;
    const bool live = e_raw < n_all;
    const long long e = live ? e_raw : n_all - 1;  // lanes past the end take part in the shuffles only
    double x[8][3];
    uint32_t nid[8];
    for (int i = 0; i < 8; ++i) {
        nid[i] = conn[8 * e + i];
        for (int d = 0; d < 3; ++d) x[i][d] = pos[3 * (long long)nid[i] + d];
    }
    const int p = part[e];
    const double youngs = mat[4 * p], nu = mat[4 * p + 1], rho = mat[4 * p + 2], hourglass = mat[4 * p + 3];
    double dnc[8][3], gc[8][3], detc;
    shape_derivatives(0.0, 0.0, 0.0, dnc);
    bool ok = reference_gradients(x, dnc, gc, &detc);
    double gam[8][4];
    for (int a = 0; a < 4; ++a) {
        double hx[3] = {0.0, 0.0, 0.0};
        for (int j = 0; j < 8; ++j)
            for (int d = 0; d < 3; ++d) hx[d] += c_modes[a][j] * x[j][d];
        for (int i = 0; i < 8; ++i) {
            double dot = hx[0] * gc[i][0] + hx[1] * gc[i][1] + hx[2] * gc[i][2];
            gam[i][a] = c_modes[a][i] - dot;
        }
    }
    const double ehg = hourglass * youngs;
    const double lam = ehg * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double mu = ehg / (2.0 * (1.0 + nu));
    // this lane's Gauss point
    const double GAUSS = 0.5773502691896258;
    const double xi = c_xi[q][0] * GAUSS, eta = c_xi[q][1] * GAUSS, zeta = c_xi[q][2] * GAUSS;
    double detj;
    double pm[4][3];
    {
        double dn[8][3], gq[8][3];
        shape_derivatives(xi, eta, zeta, dn);
        ok = reference_gradients(x, dn, gq, &detj) && ok;
        for (int b = 0; b < 4; ++b)
            for (int d = 0; d < 3; ++d) {
                double s = 0.0;
                for (int j = 0; j < 8; ++j) s += gam[j][b] * (gq[j][d] - gc[j][d]);
                pm[b][d] = s;
            }
    }
    // Column col = 3 b + e' of M (rows xx, yy, zz, xy, yz, xz; the assignments
    // of the per-element form, zeros where it leaves them).
    auto mcol = [&](int col, double t[6]) {
        const int b = col / 3, ee = col % 3;
        for (int k = 0; k < 6; ++k) t[k] = 0.0;
        if (ee == 0) {
            t[0] = pm[b][0];
            t[3] = pm[b][1];
            t[5] = pm[b][2];
        } else if (ee == 1) {
            t[1] = pm[b][1];
            t[3] = pm[b][0];
            t[4] = pm[b][2];
        } else {
            t[2] = pm[b][2];
            t[4] = pm[b][1];
            t[5] = pm[b][0];
        }
    };
    // G K G^T (upper triangle): each entry the point-ordered sum of the lanes' terms
    {
        int k = 0;
        for (int r = 0; r < 12; ++r) {
            double mr[6];
            mcol(r, mr);
            for (int cc = r; cc < 12; ++cc, ++k) {
                double mc[6], cm[6];
                mcol(cc, mc);
                cm[0] = (lam + 2.0 * mu) * mc[0] + lam * mc[1] + lam * mc[2];
                cm[1] = lam * mc[0] + (lam + 2.0 * mu) * mc[1] + lam * mc[2];
                cm[2] = lam * mc[0] + lam * mc[1] + (lam + 2.0 * mu) * mc[2];
                cm[3] = mu * mc[3];
                cm[4] = mu * mc[4];
                cm[5] = mu * mc[5];
                double s = 0.0;
                for (int t = 0; t < 6; ++t) s += mr[t] * cm[t];
                const double term = s * detj;
                double acc = 0.0;
                for (int g = 0; g < GEO_LANES; ++g) acc += __shfl_sync(0xffffffffu, term, g, GEO_LANES);
                if (q == (k & (GEO_LANES - 1))) s_gkg[grp][h_index(r, cc)] = acc;
            }
        }
    }
    // consistent mass rows and the volume, each summed over the points in order
    double nq[8];
    for (int i = 0; i < 8; ++i)
        nq[i] = 0.125 * (1.0 + c_xi[i][0] * xi) * (1.0 + c_xi[i][1] * eta) * (1.0 + c_xi[i][2] * zeta);
    double volume = 0.0;
    for (int g = 0; g < GEO_LANES; ++g) volume += __shfl_sync(0xffffffffu, detj, g, GEO_LANES);
    double lumped_i = 0.0;  // lane i < 8 keeps row i's sum
    for (int i = 0; i < 8; ++i) {
        double row = 0.0;
        for (int j = 0; j < 8; ++j) {
            const double term = rho * nq[i] * nq[j] * detj;
            double mij = 0.0;
            for (int g = 0; g < GEO_LANES; ++g) mij += __shfl_sync(0xffffffffu, term, g, GEO_LANES);
            row += mij;
        }
        if (q == i) lumped_i = row;
    }
    // every lane of the element: did any point fail?
    bool elem_ok = ok;
    for (int g = 0; g < GEO_LANES; ++g) elem_ok = __shfl_sync(0xffffffffu, (int)ok, g, GEO_LANES) != 0 && elem_ok;
    if (live && !elem_ok && q == 0) atomicExch(bad, 1);
    const long long h = hc_index[e];
    const long long sc = sc_index ? sc_index[e] : -1;
    const bool store = live && elem_ok;
    if (store) {
        lumped_out[8 * e + q] = lumped_i;
        if (q == 0) {
            volume_out[e] = volume;
            elem_mass[e] = volume * rho;
            // Material::dilatational_wave_speed, src/material.rs:226; kernel.rs:73.
            double mm = youngs * (1.0 - nu) / ((1.0 + nu) * (1.0 - 2.0 * nu));
            dt_factor[e] = (1.0 - 0.36 * nu) / sqrt(mm / rho);
        }
        if (sc >= 0) {  // an elastic element keeps its geometry in f64 (src/kernel.rs:53-91)
            const int i = q;
            for (int d = 0; d < 3; ++d) sc_geo[(SC_GRAD + 3 * i + d) * n_sc + sc] = gc[i][d];
            if (q == 0) sc_geo[SC_VOL * n_sc + sc] = volume;
            for (int aa = 0; aa < 4; ++aa) sc_geo[(SC_GAMMA + 4 * i + aa) * n_sc + sc] = gam[i][aa];
        }
    }
    // A = (ΓᵀΓ)⁻¹ by Gauss-Jordan with partial pivoting on 4x4 (every lane)
    double a[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            double s = 0.0;
            for (int i = 0; i < 8; ++i) s += gam[i][r] * gam[i][c];
            a[r][c] = s;
            a[r][4 + c] = (r == c) ? 1.0 : 0.0;
        }
    bool inv_ok = true;
    for (int k = 0; k < 4 && inv_ok; ++k) {
        int pv = k;
        for (int r = k + 1; r < 4; ++r)
            if (fabs(a[r][k]) > fabs(a[pv][k])) pv = r;
        if (a[pv][k] == 0.0) {
            inv_ok = false;
            break;
        }
        if (pv != k)
            for (int c = 0; c < 8; ++c) {
                double t = a[k][c];
                a[k][c] = a[pv][c];
                a[pv][c] = t;
            }
        double piv = a[k][k];
        for (int c = 0; c < 8; ++c) a[k][c] /= piv;
        for (int r = 0; r < 4; ++r)
            if (r != k) {
                double f = a[r][k];
                for (int c = 0; c < 8; ++c) a[r][c] -= f * a[k][c];
            }
    }
    if (store && (h >= 0 || sc >= 0) && !inv_ok && q == 0) atomicExch(bad, 2);
    __syncwarp();
    // H entries (upper triangle), split over the lanes
    for (int r = 0, k = 0; r < 12; ++r)
        for (int c = r; c < 12; ++c, ++k) {
            if ((k & (GEO_LANES - 1)) != q) continue;
            const int ar = r / 3, dr = r % 3, bc = c / 3, ec = c % 3;
            double s = 0.0;
            for (int a1 = 0; a1 < 4; ++a1)
                for (int b1 = 0; b1 < 4; ++b1) {
                    const int rr = 3 * a1 + dr, cc2 = 3 * b1 + ec;
                    s += a[ar][4 + a1] * s_gkg[grp][h_index(rr, cc2)] * a[b1][4 + bc];
                }
            s_h[grp][h_index(r, c)] = s;
        }
    __syncwarp();
    if (!store || !inv_ok || (h < 0 && sc < 0)) return;
    if (sc >= 0)
        for (int k = q; k < 78; k += GEO_LANES) sc_geo[(SC_H + k) * n_sc + sc] = s_h[grp][k];
    if (h < 0) return;
    // the element's 37 planes, split over the lanes
    for (int k = q; k < N_STATIC_PLANES; k += GEO_LANES) {
        float4 v;
        if (k < P_GRAD) {
            const int o = 4 * (k - P_CONN);
            v = make_float4(__uint_as_float(nid[o]), __uint_as_float(nid[o + 1]), __uint_as_float(nid[o + 2]), __uint_as_float(nid[o + 3]));
        } else if (k < P_GAMMA) {
            const int o = 4 * (k - P_GRAD);
            v = make_float4((float)gc[(o) / 3][(o) % 3], (float)gc[(o + 1) / 3][(o + 1) % 3], (float)gc[(o + 2) / 3][(o + 2) % 3],
                            (float)gc[(o + 3) / 3][(o + 3) % 3]);
        } else if (k < P_H) {
            const int i = k - P_GAMMA;  // gamma[4 i + a] = gam[i][a]
            v = make_float4((float)gam[i][0], (float)gam[i][1], (float)gam[i][2], (float)gam[i][3]);
        } else if (k < P_META) {
            const int o = 4 * (k - P_H);
            float f[4];
            for (int t = 0; t < 4; ++t) f[t] = o + t < 78 ? (float)s_h[grp][o + t] : 0.0f;
            v = make_float4(f[0], f[1], f[2], f[3]);
        } else {
            v = make_float4((float)volume, __uint_as_float((uint32_t)p), __uint_as_float((uint32_t)e), __uint_as_float(elem_slot[e]));
        }
        planes[k * stride + h] = v;
    }
}

// Lumped nodal masses: Σ over incident (element, corner) in element order
// (src/model.rs:268-278), and 1/m.
__global__ void k_node_masses(long long n, const uint32_t* __restrict__ off, const uint32_t* __restrict__ slot,
                              const double* __restrict__ lumped, double* __restrict__ mass, double* __restrict__ inv_mass) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double m = 0.0;
    for (uint32_t k = off[i]; k < off[i + 1]; ++k) m += lumped[slot[k]];
    mass[i] = m;
    inv_mass[i] = m > 0.0 ? 1.0 / m : 0.0;
}

__global__ void k_init_state(long long h_begin, long long n_hc, long long stride, float4* __restrict__ st) {
    long long e = h_begin + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_hc) return;
    // identity F_prev⁻¹ (0-8), identity R (9-17), zero stress, compaction, not eroded.
    const float v[28] = {1, 0, 0, 0, 1, 0, 0, 0, 1, 1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < N_STATE_PLANES; ++k) st[k * stride + e] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
}

// Node incidence of new elements [e0, e0 + ne) over their nodes [n0, n0 + nn)
// (set-up): per node its (element, corner) slots 8 e + i in increasing
// element order, the order of the reference's serial force scatter
// (src/kernel_simd.rs:573-586). Count pass: the sort keys (node) and values
// (slot) in element order, and per node its entries in all, honeycomb and
// elastic elements.
__global__ void k_incidence_count(long long e0, long long ne, long long n0, const uint32_t* __restrict__ conn,
                                  const int64_t* __restrict__ hc_index, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                                  uint32_t* __restrict__ cnt_all, uint32_t* __restrict__ cnt_hc, uint32_t* __restrict__ cnt_sc) {
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ne) return;
    const long long e = e0 + j;
    const bool honey = hc_index[e] >= 0;
    for (int i = 0; i < 8; ++i) {
        const uint32_t key = (uint32_t)(conn[8 * e + i] - n0);
        keys[8 * j + i] = key;
        vals[8 * j + i] = (uint32_t)(8 * e + i);
        atomicAdd(cnt_all + key, 1u);
        atomicAdd(honey ? cnt_hc + key : cnt_sc + key, 1u);
    }
}

// Split pass, a thread per node: its slots in element order (the stable
// sort's output at the node's offset) go to the honeycomb list (8 h + i) or
// the elastic list (8 q + i); the offsets get their global bases; the padded
// row holds the first 8 honeycomb slots (HC_ELL_MORE in front past 8).
__global__ void k_incidence_split(long long nn, const uint32_t* __restrict__ rel_all, const uint32_t* __restrict__ rel_hc,
                                  const uint32_t* __restrict__ rel_sc, uint32_t base_all, uint32_t base_hc, uint32_t base_sc,
                                  const int64_t* __restrict__ hc_index, const int64_t* __restrict__ sc_index,
                                  const uint32_t* __restrict__ all_slot, uint32_t* __restrict__ all_off, uint32_t* __restrict__ hc_off,
                                  uint32_t* __restrict__ hc_slot, uint32_t* __restrict__ sc_off, uint32_t* __restrict__ sc_slot,
                                  uint32_t* __restrict__ hc_ell) {
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j > nn) return;
    all_off[j] = base_all + rel_all[j];
    hc_off[j] = base_hc + rel_hc[j];
    sc_off[j] = base_sc + rel_sc[j];
    if (j == nn) return;
    uint32_t ph = base_hc + rel_hc[j], ps = base_sc + rel_sc[j];
    uint32_t row[8];
    int m = 0;
    for (uint32_t k = base_all + rel_all[j]; k < base_all + rel_all[j + 1]; ++k) {
        const uint32_t v = all_slot[k];
        const long long e = v >> 3;
        const uint32_t i = v & 7u;
        const long long h = hc_index[e];
        if (h >= 0) {
            const uint32_t x = (uint32_t)(8 * h + i);
            hc_slot[ph++] = x;
            if (m < 8) row[m] = x;
            ++m;
        } else {
            sc_slot[ps++] = (uint32_t)(8 * sc_index[e] + i);
        }
    }
    for (int q = m; q < 8; ++q) row[q] = HC_ELL_NONE;
    if (m > 8) row[0] = HC_ELL_MORE;
    for (int q = 0; q < 8; ++q) hc_ell[8 * j + q] = row[q];
}

// ---------------------------------------------------------------------------
// Element forces (src/kernel_simd.rs:300-491, one element per thread).
// ---------------------------------------------------------------------------
#ifndef FORCES_TPB
#define FORCES_TPB 256
#endif
#ifndef FORCES_MINB
#define FORCES_MINB 2
#endif
__device__ __forceinline__ void forces_body(const ElementArrays& el, const NodeArrays& nd, Control* ctls, int respect_done, long long e) {
    if (e >= el.n_hc) return;
    const long long S = el.stride;
    const float4 meta = ld_plane(el.planes, S, P_META, e);
    Control* ctl = ctls + __float_as_uint(meta.w);
    if (respect_done && ctl->done) return;
    float4* out = reinterpret_cast<float4*>(el.corner + 24 * e);
    const float4 st6 = el.state[6 * S + e];
    if (__float_as_uint(st6.y) != 0u) {  // already eroded: no force
        for (int k = 0; k < 6; ++k) out[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const float4 c0 = ld_plane(el.planes, S, P_CONN, e), c1 = ld_plane(el.planes, S, P_CONN + 1, e);
    const uint32_t nid[8] = {__float_as_uint(c0.x), __float_as_uint(c0.y), __float_as_uint(c0.z), __float_as_uint(c0.w),
                             __float_as_uint(c1.x), __float_as_uint(c1.y), __float_as_uint(c1.z), __float_as_uint(c1.w)};
    float grad[24];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        float4 g = ld_plane(el.planes, S, P_GRAD + k, e);
        grad[4 * k] = g.x; grad[4 * k + 1] = g.y; grad[4 * k + 2] = g.z; grad[4 * k + 3] = g.w;
    }
    float gam[32];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float4 g = ld_plane(el.planes, S, P_GAMMA + k, e);
        gam[4 * k] = g.x; gam[4 * k + 1] = g.y; gam[4 * k + 2] = g.z; gam[4 * k + 3] = g.w;
    }
    // F = Σ x_i ⊗ ∇N_i with x = (X + u) as f32; q = U Γ with u as f32.
    M3f f;
#pragma unroll
    for (int k = 0; k < 9; ++k) f.m[k] = 0.0f;
    float q[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) q[k] = 0.0f;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const long long n = nid[i];
        const double* P = nd.pos + 3 * n;
        const double* U = nd.u + 3 * n;
        const double u0 = U[0], u1 = U[1], u2 = U[2];
        const float x[3] = {(float)(__ldg(P) + u0), (float)(__ldg(P + 1) + u1), (float)(__ldg(P + 2) + u2)};
        const float ul[3] = {(float)u0, (float)u1, (float)u2};
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int c = 0; c < 3; ++c) f.m[3 * a + c] = x[a] * grad[3 * i + c] + f.m[3 * a + c];
#pragma unroll
        for (int mode = 0; mode < 4; ++mode)
#pragma unroll
            for (int dir = 0; dir < 3; ++dir) q[3 * mode + dir] = ul[dir] * gam[4 * i + mode] + q[3 * mode + dir];
    }
    const float det = det3(f);
    if (det <= 0.0f) {  // inverted: erode (src/kernel_simd.rs:324-331)
        el.state[6 * S + e] = make_float4(st6.x, __uint_as_float(1u), st6.z, st6.w);
        el.eroded_all[__float_as_uint(meta.z)] = 1;
        atomicAdd(reinterpret_cast<unsigned long long*>(&ctl->eroded_step), 1ull);
        for (int k = 0; k < 6; ++k) out[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    float st[28];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        float4 s4 = __ldcs(el.state + k * S + e);
        st[4 * k] = s4.x; st[4 * k + 1] = s4.y; st[4 * k + 2] = s4.z; st[4 * k + 3] = s4.w;
    }
    st[24] = st6.x; st[25] = st6.y; st[26] = st6.z; st[27] = st6.w;
    const MaterialF32& mat = el.mats[__float_as_uint(meta.y)];
    M3f tau, f_inv;
    honeycomb_update(f, det, st, mat, tau, f_inv);
#pragma unroll
    for (int k = 0; k < 7; ++k) __stcs(el.state + k * S + e, make_float4(st[4 * k], st[4 * k + 1], st[4 * k + 2], st[4 * k + 3]));
    // f_i = τ F⁻ᵀ ∇N_i V₀
    M3f m;
    mat_mul_t(tau, f_inv, m);
    const float vol = meta.x;
#pragma unroll
    for (int k = 0; k < 9; ++k) m.m[k] = m.m[k] * vol;
    float fo[24];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float acc = m.m[3 * a] * grad[3 * i];
            acc = m.m[3 * a + 1] * grad[3 * i + 1] + acc;
            acc = m.m[3 * a + 2] * grad[3 * i + 2] + acc;
            fo[3 * i + a] = acc;
        }
    // Hourglass: rr = H q (column order), f += rr Γᵀ.
    float hsym[80];
#pragma unroll
    for (int k = 0; k < 20; ++k) {
        float4 h4 = ld_plane(el.planes, S, P_H + k, e);
        hsym[4 * k] = h4.x; hsym[4 * k + 1] = h4.y; hsym[4 * k + 2] = h4.z; hsym[4 * k + 3] = h4.w;
    }
    float rr[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) rr[k] = 0.0f;
#pragma unroll
    for (int col = 0; col < 12; ++col)
#pragma unroll
        for (int row = 0; row < 12; ++row) rr[row] = hsym[h_index(row, col)] * q[col] + rr[row];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int dir = 0; dir < 3; ++dir) {
            float acc = fo[3 * i + dir];
#pragma unroll
            for (int mode = 0; mode < 4; ++mode) acc = rr[3 * mode + dir] * gam[4 * i + mode] + acc;
            fo[3 * i + dir] = acc;
        }
#pragma unroll
    for (int k = 0; k < 6; ++k) out[k] = make_float4(fo[4 * k], fo[4 * k + 1], fo[4 * k + 2], fo[4 * k + 3]);
}

// Nodal internal force, component d: ordered f64 sum of the incident corner
// forces (element order). Up to 8 corners (every node of a structured hex
// mesh) the loads are all issued before the sum.
// The node's slots come from its padded row of 8 (one round of loads
// before the corner loads); a node with more than 8 uses the CSR.
__device__ __forceinline__ double gather_component(const NodeArrays& nd, const float* __restrict__ corner, long long n, int d) {
    const uint4 r0 = __ldg(nd.hc_ell + 2 * n), r1 = __ldg(nd.hc_ell + 2 * n + 1);
    double f = 0.0;
    if (r0.x != HC_ELL_MORE) {
        const uint32_t sl[8] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w};
        float c[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) c[j] = sl[j] != HC_ELL_NONE ? __ldg(corner + 3ull * sl[j] + d) : 0.f;  // slot = 8 e + corner
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if (sl[j] != HC_ELL_NONE) f += (double)c[j];
    } else {
        const uint32_t b = __ldg(nd.hc_off + n), m = __ldg(nd.hc_off + n + 1) - b;
        for (uint32_t k = 0; k < m; ++k) f += (double)__ldg(corner + 3ull * __ldg(nd.hc_slot + b + k) + d);
    }
    return f;
}
__device__ __forceinline__ void gather_node(const NodeArrays& nd, const float* __restrict__ corner, long long n,
                                            double& fx, double& fy, double& fz) {
    fx = gather_component(nd, corner, n, 0);
    fy = gather_component(nd, corner, n, 1);
    fz = gather_component(nd, corner, n, 2);
}

// queue == nullptr: grid-stride over the active chunks. Otherwise a
// persistent grid whose blocks take active chunks from queue[0] one at a
// time, so a block that starts late (its SM busy with other streams' work)
// takes fewer chunks instead of finishing late; the last block to finish
// (queue[1] counts them) sets both counters back to zero.
__global__ void __launch_bounds__(FORCES_TPB, FORCES_MINB) k_forces(ElementArrays el, NodeArrays nd, Control* ctls, int respect_done,
                                                                    unsigned* queue) {
    if (!queue) {
        FOR_ACTIVE(el.act_hc, el.n_hc, 1, g) {
            int lane;
            forces_body(el, nd, ctls, respect_done, active_entity(el.act_hc, g, 1, &lane));
        }
        return;
    }
    const long long chunks = active_total(el.act_hc, el.n_hc, 1) / CHUNK;
    __shared__ long long s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = (long long)atomicAdd(queue, 1u);
        __syncthreads();
        const long long item = s_item;
        __syncthreads();
        if (item >= chunks) break;
        for (int t = threadIdx.x; t < CHUNK; t += FORCES_TPB) {
            int lane;
            forces_body(el, nd, ctls, respect_done, active_entity(el.act_hc, item * CHUNK + t, 1, &lane));
        }
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(queue + 1, 1u) == gridDim.x - 1) {
            queue[0] = 0u;
            queue[1] = 0u;
        }
    }
}

// Elastic elements: the reference's scalar f64 element (src/kernel.rs:116-156)
// with the Hencky stress, one element per thread: F = Σ x_i ⊗ ∇N_i at
// x = X + u; det F <= 0 erodes the element; f_i = (τ F⁻ᵀ V) ∇N_i plus the
// hourglass force R Γᵀ with R = H (U Γ). Corner forces in f64.
constexpr int SC_TPB = 128;
__device__ __forceinline__ void scalar_force_body(const ElementArrays& el, const NodeArrays& nd, Control* ctls, int respect_done,
                                                  long long i) {
    if (i >= el.sc_count) return;
    const long long e = el.sc_model[i];
    Control* ctl = ctls + el.elem_slot[e];
    if (respect_done && ctl->done) return;
    double* out = el.sc_corner + 24 * i;
    if (el.eroded_all[e]) {
        for (int k = 0; k < 24; ++k) out[k] = 0.0;
        return;
    }
    const long long S = el.sc_stride;
    const double* G = el.sc_geo;
    // One pass over the nodes accumulates F (x = X + u) and q = U Γ, in the
    // order of the all-node loops; ∇N and Γ rows are read again below, so
    // no per-node arrays stay live (the kernel's occupancy is register-bound).
    double f[9], q[12];
    for (int k = 0; k < 9; ++k) f[k] = 0.0;
    for (int k = 0; k < 8; ++k) {
        const long long n = el.conn_all[8 * e + k];
        double xk[3], uk[3], gk[3], ak[4];
        for (int d = 0; d < 3; ++d) {
            uk[d] = nd.u[3 * n + d];
            xk[d] = nd.pos[3 * n + d] + uk[d];
            gk[d] = G[(SC_GRAD + 3 * k + d) * S + i];
        }
        for (int a = 0; a < 4; ++a) ak[a] = G[(SC_GAMMA + 4 * k + a) * S + i];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) f[3 * a + b] += xk[a] * gk[b];
        for (int a = 0; a < 4; ++a)
            for (int d = 0; d < 3; ++d) q[3 * a + d] = k == 0 ? uk[d] * ak[a] : q[3 * a + d] + uk[d] * ak[a];
    }
    if (det3d(f) <= 0.0) {
        el.eroded_all[e] = 1;
        atomicAdd(reinterpret_cast<unsigned long long*>(&ctl->eroded_step), 1ull);
        for (int k = 0; k < 24; ++k) out[k] = 0.0;
        return;
    }
    double tau[9], finv[9];
    hencky_elastic(el.sc_mat[2 * i], el.sc_mat[2 * i + 1], f, tau);
    inv3d(f, finv);
    const double vol = G[SC_VOL * S + i];
    double m[9];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            double t = tau[3 * a] * finv[3 * b];
            t = t + tau[3 * a + 1] * finv[3 * b + 1];
            t = t + tau[3 * a + 2] * finv[3 * b + 2];
            m[3 * a + b] = t * vol;
        }
    double r[12];
    for (int row = 0; row < 12; ++row) {
        double t = G[(SC_H + h_index(0, row)) * S + i] * q[0];
        for (int c = 1; c < 12; ++c) t = t + G[(SC_H + (row <= c ? h_index(row, c) : h_index(c, row))) * S + i] * q[c];
        r[row] = t;
    }
    // f_i = (τ F⁻ᵀ V) ∇N_i plus the hourglass force (R Γᵀ)_i
    for (int k = 0; k < 8; ++k) {
        double gk[3], ak[4];
        for (int d = 0; d < 3; ++d) gk[d] = G[(SC_GRAD + 3 * k + d) * S + i];
        for (int a = 0; a < 4; ++a) ak[a] = G[(SC_GAMMA + 4 * k + a) * S + i];
        for (int d = 0; d < 3; ++d) {
            double o = m[3 * d] * gk[0];
            o = o + m[3 * d + 1] * gk[1];
            o = o + m[3 * d + 2] * gk[2];
            double t = r[d] * ak[0];
            for (int a = 1; a < 4; ++a) t = t + r[3 * a + d] * ak[a];
            out[3 * k + d] = o + t;
        }
    }
}

__global__ void __launch_bounds__(SC_TPB) k_forces_scalar(ElementArrays el, NodeArrays nd, Control* ctls, int respect_done) {
    FOR_ACTIVE(el.act_sc, el.n_sc, 1, g) {
        int lane;
        const long long t = active_entity(el.act_sc, g, 1, &lane);
        // a run lists the elastic elements with a free node; drop-in calls take them all
        scalar_force_body(el, nd, ctls, respect_done, el.sc_list ? (t < el.n_sc ? (long long)el.sc_list[t] : el.sc_count) : t);
    }
}

// The elastic elements' corner forces on node n, component d, added to f in
// element order after the honeycomb ones (src/kernel.rs:192-201 adds the
// scalar elements after the lane blocks' scatter).
__device__ __forceinline__ double add_scalar_corners(const ElementArrays& el, const NodeArrays& nd, long long n, int d, double f) {
    const uint32_t b = nd.sc_off[n], m = nd.sc_off[n + 1] - b;
    for (uint32_t k = 0; k < m; ++k) f += el.sc_corner[3ull * nd.sc_slot[b + k] + d];
    return f;
}

__global__ void k_gather(ElementArrays el, NodeArrays nd, double* __restrict__ f_out) {
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nd.n) return;
    double fx, fy, fz;
    gather_node(nd, el.corner, n, fx, fy, fz);
    if (el.n_sc > 0) {
        fx = add_scalar_corners(el, nd, n, 0, fx);
        fy = add_scalar_corners(el, nd, n, 1, fy);
        fz = add_scalar_corners(el, nd, n, 2, fz);
    }
    f_out[3 * n] = fx;
    f_out[3 * n + 1] = fy;
    f_out[3 * n + 2] = fz;
}

// Half step: v½ = v + ½dt (f_ext - f_int)/m ; u += dt v½ ; fixed -> 0 (src/solver.rs:314-323).
// Thread per node component d: the loads are issued before the crash's
// done flag is known (they are harmless), so one latency covers them all.
__device__ __forceinline__ void half_body(const NodeArrays& nd, const Control* ctls, long long n, int d) {
    if (n >= nd.n) return;
    const long long k = 3 * n + d;
    const int slot = nd.node_slot[n];
    const double fe = nd.f_ext[k], fi = nd.f_int[k], v = nd.v[k], u0 = nd.u[k], im = nd.inv_mass[n];
    const bool fixed = nd.fixed[n] != 0;
    const Control* ctl = ctls + slot;
    if (ctl->done) return;
    const double dt = step_dt(ctl);
    const double a = (fe - fi) * im;
    double vh = v + 0.5 * dt * a;
    double u = u0 + dt * vh;
    if (fixed) {
        u = 0.0;
        vh = 0.0;
        nd.v[k] = 0.0;
    }
    nd.v_half[k] = vh;
    nd.u[k] = u;
}

__global__ void k_half(NodeArrays nd, Control* ctls) {
    FOR_ACTIVE(nd.act_node, nd.n, 3, g) {
        int d;
        const long long n = active_entity(nd.act_node, g, 3, &d);
        half_body(nd, ctls, n, d);
    }
}

// Full step with the fused force gather: v = (v½ + ½dt a) damping (src/solver.rs:334-342).
// Thread per node component d, loads issued before the done flag is known.
__device__ __forceinline__ void full_body(const ElementArrays& el, const NodeArrays& nd, const Control* ctls, long long n, int d) {
    if (n >= nd.n) return;
    const long long k = 3 * n + d;
    const int slot = nd.node_slot[n];
    const double fe = nd.f_ext[k], vh = nd.v_half[k], im = nd.inv_mass[n];
    const bool fixed = nd.fixed[n] != 0;
    double f = gather_component(nd, el.corner, n, d);
    if (el.n_sc > 0) f = add_scalar_corners(el, nd, n, d, f);
    const Control* ctl = ctls + slot;
    if (ctl->done) return;
    const double dt = step_dt(ctl);
    const double a = (fe - f) * im;
    const double v = (vh + 0.5 * dt * a) * ctl->damping;
    nd.v[k] = fixed ? 0.0 : v;
    nd.f_int[k] = f;
}

__global__ void k_full(ElementArrays el, NodeArrays nd, Control* ctls) {
    FOR_ACTIVE(nd.act_node, nd.n, 3, g) {
        int d;
        const long long n = active_entity(nd.act_node, g, 3, &d);
        full_body(el, nd, ctls, n, d);
    }
}

// One step's full update fused with the next step's half step
// (src/solver.rs:334-342, then :314-323 of the next step), thread per node
// component: the ordered corner gather gives f_int at the new positions,
// v = (v½ + ½dt a) damping; then, unless this step is the crash's last by
// its step count or end time, the next step's v½ = v + ½dt' (f_ext' - f_int)/m
// and u += dt' v½ with the next step's dt' and contact forces f_ext'. The
// arithmetic is that of full_body followed by half_body; fixed DOFs are zero
// as there. A crash that stops here keeps u and v½ of this step. Neither v
// nor f_int is read before the next full update rewrites them (the next
// half step is done here; a step followed by a check or record is never
// fused), so they are stored only for a crash that stops here.
__device__ __forceinline__ void fused_body(const ElementArrays& el, const NodeArrays& nd, const Control* ctls, long long n, int d) {
    if (n >= nd.n) return;
    const long long k = 3 * n + d;
    const int slot = nd.node_slot[n];
    const double fe = nd.f_ext[k], fe1 = nd.f_ext_next[k], vh = nd.v_half[k], u0 = nd.u[k], im = nd.inv_mass[n];
    const bool fixed = nd.fixed[n] != 0;
    double f = gather_component(nd, el.corner, n, d);
    if (el.n_sc > 0) f = add_scalar_corners(el, nd, n, d, f);
    const Control* ctl = ctls + slot;
    if (ctl->done) return;
    const double dt = step_dt(ctl);
    const double a = (fe - f) * im;
    const double v = fixed ? 0.0 : (vh + 0.5 * dt * a) * ctl->damping;
    if (last_step_by_count_or_time(ctl)) {
        nd.v[k] = v;
        nd.f_int[k] = f;
        return;
    }
    const double dt1 = next_step_dt(ctl);
    const double a1 = (fe1 - f) * im;
    double vh1 = v + 0.5 * dt1 * a1;
    double u1 = u0 + dt1 * vh1;
    if (fixed) {
        u1 = 0.0;
        vh1 = 0.0;
    }
    nd.v_half[k] = vh1;
    nd.u[k] = u1;
}

__device__ void step_end_slot(Control* ctl, int sl, const ContactArrays& ca, const VehicleArrays& va, int check_separation);

// The fused pass, then the step's end (k_step_end without the reduction stop
// rules, which no fused step has) run by the last block to finish: every
// other block has read the control blocks by then.
__global__ void k_fused(ElementArrays el, NodeArrays nd, Control* ctls, ContactArrays ca, VehicleArrays va, int* __restrict__ done_out,
                        int* __restrict__ mass_flag, unsigned* __restrict__ counter) {
    FOR_ACTIVE(nd.act_node, nd.n, 3, g) {
        int d;
        const long long n = active_entity(nd.act_node, g, 3, &d);
        fused_body(el, nd, ctls, n, d);
    }
    __shared__ int s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(counter, 1u) == gridDim.x - 1 ? 1 : 0;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x == 0) {
        *mass_flag = 0;
        *counter = 0;
    }
    for (int sl = threadIdx.x; sl < ca.n_slots; sl += blockDim.x) {
        Control* ctl = ctls + sl;
        if (!ctl->done) step_end_slot(ctl, sl, ca, va, 0);
        done_out[sl] = ctl->done;
    }
}

// ---------------------------------------------------------------------------
// Stable time step (src/kernel.rs:207-237, src/element.rs:176-186) and the
// per-element added mass of selective mass scaling (src/kernel.rs:243-258).
// ---------------------------------------------------------------------------
__device__ void char_length_and_volume(const double p[8][3], double* l, double* vol_out) {
    const int TETS[6][4] = {{0, 1, 2, 6}, {0, 2, 3, 6}, {0, 3, 7, 6}, {0, 7, 4, 6}, {0, 4, 5, 6}, {0, 5, 1, 6}};
    const int FACES[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}};
    double vol = 0.0;
#pragma unroll
    for (int t = 0; t < 6; ++t) {
        const double* a = p[TETS[t][0]];
        double e1[3], e2[3], e3[3];
        for (int d = 0; d < 3; ++d) {
            e1[d] = p[TETS[t][1]][d] - a[d];
            e2[d] = p[TETS[t][2]][d] - a[d];
            e3[d] = p[TETS[t][3]][d] - a[d];
        }
        double cx = e1[1] * e2[2] - e1[2] * e2[1];
        double cy = e1[2] * e2[0] - e1[0] * e2[2];
        double cz = e1[0] * e2[1] - e1[1] * e2[0];
        vol = vol + (cx * e3[0] + cy * e3[1] + cz * e3[2]) / 6.0;
    }
    double a_max = 0.0;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        double d1[3], d2[3];
        for (int d = 0; d < 3; ++d) {
            d1[d] = p[FACES[f][2]][d] - p[FACES[f][0]][d];
            d2[d] = p[FACES[f][3]][d] - p[FACES[f][1]][d];
        }
        double cx = d1[1] * d2[2] - d1[2] * d2[1];
        double cy = d1[2] * d2[0] - d1[0] * d2[2];
        double cz = d1[0] * d2[1] - d1[1] * d2[0];
        double a = 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
        a_max = fmax(a_max, a);
    }
    *vol_out = vol;
    *l = (vol <= 0.0 || a_max <= 0.0) ? CUDART_INF : vol / a_max;
}

constexpr int DT_TPB = 256;

// Per-element stability limit and mass-scaling surplus. The minimum per crash
// slot is an atomicMin on the bit pattern of a non-negative double (order
// independent); lanes of a warp that share a slot reduce first.
__device__ __forceinline__ void elem_dt_body(const ElementArrays& el, const NodeArrays& nd, Control* ctls, const double* __restrict__ u,
                                             int respect_done, long long e) {
    const int lane = threadIdx.x & 31;
    uint32_t slot = 0xffffffffu;
    double dt = CUDART_INF, extra = 0.0;
    if (e < el.n_all) {
        // Loads that do not depend on the crash's done flag go first.
        slot = el.elem_slot[e];
        const bool eroded = el.eroded_all[e] != 0;
        const uint4 q0 = __ldg(reinterpret_cast<const uint4*>(el.conn_all + 8 * e));
        const uint4 q1 = __ldg(reinterpret_cast<const uint4*>(el.conn_all + 8 * e) + 1);
        Control* ctl = ctls + slot;
        if (respect_done && ctl->done) {
            slot = 0xffffffffu;
        } else {
            if (!eroded) {
                const uint32_t conn[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
                double p[8][3];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const long long n = conn[i];
                    for (int d = 0; d < 3; ++d) p[i][d] = nd.pos[3 * n + d] + u[3 * n + d];
                }
                double l, vol;
                char_length_and_volume(p, &l, &vol);
                if (isfinite(l) && vol > 0.0) dt = l * el.dt_factor[e];
            }
            const double floor = ctl->dt_floor;
            if (dt < floor) {
                double r = floor / dt;
                extra = (fmin(r * r, 100.0) - 1.0) * el.elem_mass[e];
            }
            el.elem_dt[e] = dt;
            el.elem_extra[e] = extra;
        }
    }
    const uint32_t s0 = __shfl_sync(0xffffffffu, slot, 0);
    const bool uniform = __all_sync(0xffffffffu, slot == s0);
    if (uniform) {
        if (s0 == 0xffffffffu) return;
        for (int off = 16; off > 0; off >>= 1) {
            dt = fmin(dt, __shfl_down_sync(0xffffffffu, dt, off));
            extra += __shfl_down_sync(0xffffffffu, extra, off);
        }
        if (lane == 0) {
            atomicMin(&ctls[s0].dt_stable_bits, (unsigned long long)__double_as_longlong(dt));
            if (extra > 0.0) atomicAdd(&ctls[s0].added_total_acc, extra);
        }
    } else if (slot != 0xffffffffu) {
        atomicMin(&ctls[slot].dt_stable_bits, (unsigned long long)__double_as_longlong(dt));
        if (extra > 0.0) atomicAdd(&ctls[slot].added_total_acc, extra);
    }
}

__global__ void __launch_bounds__(DT_TPB) k_elem_dt(ElementArrays el, NodeArrays nd, Control* ctls, const double* __restrict__ u,
                                                    int respect_done, long long e_begin) {
    FOR_ACTIVE(el.act_all, el.n_all - e_begin, 1, g) {
        int lane;
        elem_dt_body(el, nd, ctls, u, respect_done, e_begin + active_entity(el.act_all, g, 1, &lane));
    }
}

// The adaptive step decision of src/solver.rs:288-299, one thread per slot.
__global__ void k_dt_finalize(Control* ctls, int n_slots, int* __restrict__ mass_flag) {
    const int sl = blockIdx.x * blockDim.x + threadIdx.x;
    if (sl >= n_slots) return;
    Control* ctl = ctls + sl;
    if (ctl->done) return;
    const double dt_stable = __longlong_as_double((long long)ctl->dt_stable_bits);
    const double total = ctl->added_total_acc;
    ctl->dt_stable_bits = (unsigned long long)__double_as_longlong(CUDART_INF);
    ctl->added_total_acc = 0.0;
    if (!isfinite(dt_stable)) return;
    double dt_use = dt_stable;
    if (ctl->dt_floor > 0.0 && dt_stable < ctl->dt_floor) {
        ctl->mass_scale_now = 1;
        *mass_flag = 1;  // some crash scales its masses this step
        ctl->added_total = total;
        ctl->added_mass_max = fmax(ctl->added_mass_max, total);
        dt_use = ctl->dt_floor;
    }
    ctl->dt_cfl = ctl->dt_scale * fmin(dt_use, ctl->contact_dt);
}

// Added nodal mass (element order, src/kernel.rs:246-255) and 1/(m + added).
__device__ __forceinline__ void mass_scaling_body(const ElementArrays& el, const NodeArrays& nd, const Control* ctls, int force_apply,
                                                  long long n) {
    if (n >= nd.n || (!force_apply && !*nd.mass_flag)) return;
    const Control* ctl = ctls + nd.node_slot[n];
    if (!force_apply && (ctl->done || !ctl->mass_scale_now)) return;
    const double floor = ctl->dt_floor;
    double add = 0.0;
    for (uint32_t k = nd.all_off[n]; k < nd.all_off[n + 1]; ++k) {
        uint32_t e = nd.all_slot[k] >> 3;
        if (el.elem_dt[e] < floor) add += el.elem_extra[e] / 8.0;
    }
    nd.added[n] = add;
    const double m = nd.mass[n] + add;
    nd.inv_mass[n] = m > 0.0 ? 1.0 / m : 0.0;
}

__global__ void k_mass_scaling(ElementArrays el, NodeArrays nd, Control* ctls, int force_apply) {
    FOR_ACTIVE(nd.act_node, nd.n, 1, g) {
        int lane;
        mass_scaling_body(el, nd, ctls, force_apply, active_entity(nd.act_node, g, 1, &lane));
    }
}

__global__ void k_nonfinite(NodeArrays nd, Control* ctls) {
    FOR_ACTIVE(nd.act_node, nd.n, 1, g) {
        int lane;
        const long long n = active_entity(nd.act_node, g, 1, &lane);
        if (n >= nd.n) continue;
        Control* ctl = ctls + nd.node_slot[n];
        if (ctl->done) continue;
        if (!isfinite(nd.u[3 * n]) || !isfinite(nd.u[3 * n + 1]) || !isfinite(nd.u[3 * n + 2])) ctl->nonfinite = 1;
    }
}

// The active chunk lists: thread per chunk (all entity spaces), a chunk is
// active while any crash slot it holds is still running. One atomic per warp
// and space.
__global__ void k_build_active(ActiveBuild b, const Control* __restrict__ ctls) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    int space = -1;
    bool alive = false;
    if (t < b.n_chunks) {
        space = 0;
        while (space + 1 < ACTIVE_SPACES && t >= b.space_off[space + 1]) ++space;
        for (int k = b.chunk_lo[t]; k <= b.chunk_hi[t] && !alive; ++k) alive = !ctls[k].done;
    }
    const unsigned want = __ballot_sync(0xffffffffu, alive);
    const unsigned same = __match_any_sync(0xffffffffu, space);
    const unsigned grp = want & same;
    if (alive) {
        const int leader = __ffs(grp) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(&b.counts[space], __popc(grp));
        base = __shfl_sync(grp, base, leader);
        b.lists[b.space_off[space] + base + __popc(grp & ((1u << lane) - 1u))] = (int)(t - b.space_off[space]);
    }
}

// End of a step (src/solver.rs:344-345 plus the stop rules), one thread per slot.
__device__ void step_end_slot(Control* ctl, int sl, const ContactArrays& ca, const VehicleArrays& va, int check_separation);

// One thread per slot; also mirrors each slot's done flag into done_out (a
// compact array the host polls).
__global__ void k_step_end(Control* ctls, ContactArrays ca, VehicleArrays va, int check_separation, int* __restrict__ done_out,
                           int* __restrict__ mass_flag) {
    const int sl = blockIdx.x * blockDim.x + threadIdx.x;
    if (sl == 0) *mass_flag = 0;  // the step's mass scaling is done
    if (sl >= ca.n_slots) return;
    Control* ctl = ctls + sl;
    if (!ctl->done) step_end_slot(ctl, sl, ca, va, check_separation);
    done_out[sl] = ctl->done;
}

__device__ void step_end_slot(Control* ctl, int sl, const ContactArrays& ca, const VehicleArrays& va, int check_separation) {
    const double dt = step_dt(ctl);
    ctl->step += 1;
    ctl->t = ctl->t + dt;
    ctl->dt_min = fmin(ctl->dt_min, dt);
    ctl->eroded_total += ctl->eroded_step;
    ctl->eroded_step = 0;
    ctl->mass_scale_now = 0;
    int hit = 0;
    for (int c = ca.slot_contact_off[sl]; c < ca.slot_contact_off[sl + 1]; ++c) {
        if (ca.counts_for_stop[c] && ca.pen_count[c] > 0) hit = 1;
        ca.pen_count[c] = 0;
        ca.pen_max_bits[c] = 0;
    }
    if (hit) ctl->last_hit = ctl->step - 1;
    if (ctl->nonfinite) {
        ctl->done = 1;
        ctl->status = -2;  // CRUSH_ERR_NONFINITE
        return;
    }
    if (ctl->copy_timeout) {
        ctl->done = 1;
        ctl->status = -4;  // CRUSH_ERR_TIMEOUT
        return;
    }
    if (ctl->max_steps > 0 && ctl->step >= ctl->max_steps) ctl->done = 1;
    if (!(ctl->t < ctl->end_time)) ctl->done = 1;
    if (check_separation) {
        for (int veh = 0; veh < 2; ++veh) {
            double m = 0.0, p = 0.0;
            for (int b = 0; b < va.vx_blocks; ++b) {
                m += ctl->vx_part[veh][b][0];
                p += ctl->vx_part[veh][b][1];
            }
            ctl->vx[veh] = m > 0.0 ? p / m : 0.0;
        }
        if (ctl->stop_rule == 1 && ctl->step % 10 == 0 && ctl->last_hit >= 0 && ctl->step - 1 - ctl->last_hit >= 100 &&
            ctl->vx[1] - ctl->vx[0] >= 0.0)
            ctl->done = 1;
    }
}

// ---------------------------------------------------------------------------
// Node-to-face penalty contact (src/contact.rs:92-160): face geometry, a
// broad phase (a hierarchical hashed grid rebuilt every step for moving
// faces, an exact grid built once for static ones), first-hit (minimum face
// index) search per primary node, and an ordered gather of the reactions.
// ---------------------------------------------------------------------------

// Grid cells a box covers at cell size cs. False when the box is not finite
// or covers more than `budget` cells; each axis range is checked before any
// product, so a loop over the returned range is always short.
__device__ __forceinline__ bool box_cells(const double* lo, const double* hi, double cs, long long* r, int budget) {
    for (int d = 0; d < 3; ++d)
        if (!isfinite(lo[d]) || !isfinite(hi[d]) || !(lo[d] <= hi[d])) return false;
    const double lim = 4.0e15;  // cell coordinates stay exact in f64 and far from long long overflow
    double a[6];
    for (int d = 0; d < 3; ++d) {
        a[2 * d] = floor(lo[d] / cs);
        a[2 * d + 1] = floor(hi[d] / cs);
        if (fabs(a[2 * d]) > lim || fabs(a[2 * d + 1]) > lim) return false;
    }
    double prod = 1.0;
    for (int d = 0; d < 3; ++d) {
        const double span = a[2 * d + 1] - a[2 * d];
        if (span < 0.0 || span >= budget) return false;
        prod *= span + 1.0;
    }
    if (prod > budget) return false;
    for (int k = 0; k < 6; ++k) r[k] = (long long)a[k];
    return true;
}

// Hash of the cell of a point (any finite coordinates; non-finite points map
// to cell 0) at cell size cs and grid level `level`.
__device__ __forceinline__ unsigned point_cell_hash(const double* p, double cs, int level) {
    long long q[3];
    for (int d = 0; d < 3; ++d) {
        double a = floor(p[d] / cs);
        q[d] = (isfinite(a) && fabs(a) <= 4.0e15) ? (long long)a : 0;
    }
    return cell_hash(q[0], q[1], q[2], level);
}

// Face geometry (src/contact.rs:95-110) at X + u.
__device__ __forceinline__ void face_geometry(const ContactArrays& ca, const NodeArrays& nd, long long f, double md, FaceGeo& g) {
    for (int k = 0; k < 4; ++k) {
        long long n = ca.faces[4 * f + k];
        for (int d = 0; d < 3; ++d) g.x[k][d] = nd.pos[3 * n + d] + nd.u[3 * n + d];
    }
    double e1[3], e2[3];
    for (int d = 0; d < 3; ++d) {
        e1[d] = g.x[1][d] - g.x[0][d];
        e2[d] = g.x[2][d] - g.x[0][d];
    }
    double nx = e1[1] * e2[2] - e1[2] * e2[1];
    double ny = e1[2] * e2[0] - e1[0] * e2[2];
    double nz = e1[0] * e2[1] - e1[1] * e2[0];
    double len = sqrt(nx * nx + ny * ny + nz * nz);
    g.n[0] = nx / len; g.n[1] = ny / len; g.n[2] = nz / len;
    for (int d = 0; d < 3; ++d) {
        g.c[d] = (((g.x[0][d] + g.x[1][d]) + g.x[2][d]) + g.x[3][d]) / 4.0;
        double lo = g.x[0][d], hi = g.x[0][d];
        for (int k = 1; k < 4; ++k) {
            lo = fmin(lo, g.x[k][d]);
            hi = fmax(hi, g.x[k][d]);
        }
        g.lo[d] = lo + -md;
        g.hi[d] = hi + md;
    }
}

// The grid level and cell range of a face's key box (klo, khi) in contact
// c: returns the level, GRID_LEVELS for a big face, -1 for no insertion.
__device__ __forceinline__ int box_level(const ContactArrays& ca, int c, const double* klo, const double* khi, long long* r) {
    if (klo[0] > khi[0] || klo[1] > khi[1] || klo[2] > khi[2]) return -1;  // no point can hit the face
    double cs = ca.cell[c];
    for (int level = 0; level < GRID_LEVELS; ++level, cs *= 4.0)
        if (box_cells(klo, khi, cs, r, LEVEL_CELL_BUDGET)) return level;
    return GRID_LEVELS;
}

// Thread per face: the face's geometry at X + u. The faces are
// face_list[0, n) when face_list is given (the run: moving faces only), else
// face_off[c0] + [0, n).
// FACE_LANES lanes per face: its geometry at X + u, and — when the search
// builds the dynamic grids (do_grid) and the face's contact has one — its key
// box (lane t takes triangle t, the quad combines them), grid level and
// cells, stored for the fill pass, with one count per cell added to the
// cell's bucket (the lanes split the cells); a face whose box fits no level
// is listed as a big face with its key box. Every face of a grid contact that
// the pass visits gets its cell record (level -1: no inserts), so the fill
// pass, over the same faces, inserts exactly what was counted.
constexpr int FACE_LANES = 4;
__device__ __forceinline__ void contact_face_body(const ContactArrays& ca, const NodeArrays& nd, const Control* ctls, int c0,
                                                  const uint32_t* __restrict__ face_list, long long n, int run_mode, int do_grid,
                                                  long long t, int lane) {
    if (t >= n) return;  // uniform over the face's lanes, as is every branch before the shuffles
    const unsigned qmask = 0xFu << (threadIdx.x & 28u);
    const long long f = face_list ? (long long)face_list[t] : ca.face_off[c0] + t;
    const int c = ca.face_contact[f];
    const int tab = ca.tab_off[c];
    const bool grid = do_grid && ca.tab_off[c + 1] > tab;
    if (run_mode && ctls[ca.contact_slot[c]].done) {
        if (grid && lane == 0) ca.cells[f].level = -1;
        return;
    }
    const double md = ca.max_distance[c];
    FaceGeo g;
    face_geometry(ca, nd, f, md, g);
    {
        constexpr int per = (int)(sizeof(FaceGeo) / sizeof(double)) / FACE_LANES;
        const double* src = reinterpret_cast<const double*>(&g);
        double* dst = reinterpret_cast<double*>(ca.geo + f);
#pragma unroll
        for (int k = 0; k < (int)(sizeof(FaceGeo) / sizeof(double)); ++k)
            if (k / per == lane) dst[k] = src[k];
    }
    if (!grid) return;
    double rlo[3] = {1e300, 1e300, 1e300}, rhi[3] = {-1e300, -1e300, -1e300};
    int perp = key_box_triangle(g.x, g.n, g.c, lane, rlo, rhi) == KEY_TRI_PERP ? 1 : 0;
#pragma unroll
    for (int off = 1; off < FACE_LANES; off <<= 1) {
        perp |= __shfl_xor_sync(qmask, perp, off, FACE_LANES);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            rlo[d] = fmin(rlo[d], __shfl_xor_sync(qmask, rlo[d], off, FACE_LANES));
            rhi[d] = fmax(rhi[d], __shfl_xor_sync(qmask, rhi[d], off, FACE_LANES));
        }
    }
    double klo[3], khi[3];
    key_box_finish(g.x, g.n, md, perp != 0, rlo, rhi, klo, khi);
    long long r[6];
    const int level = box_level(ca, c, klo, khi, r);
    FaceCells fc;
    fc.level = level;
    fc.lo[0] = r[0];
    fc.lo[1] = r[2];
    fc.lo[2] = r[4];
    fc.span[0] = fc.span[1] = fc.span[2] = 0;
    if (level == GRID_LEVELS) {
        if (lane == 0) {
            // A face is listed at most once per search and the list holds
            // every face of the grid contacts, so it cannot overrun.
            const int slot = atomicAdd(ca.big_count, 1);
            if (slot < ca.big_cap) {
                ca.big_faces[slot] = (uint32_t)f;
                for (int d = 0; d < 3; ++d) {
                    ca.big_box[6 * (long long)slot + d] = klo[d];
                    ca.big_box[6 * (long long)slot + 3 + d] = khi[d];
                }
            }
            atomicAdd(&ca.search_stats[3 * c + 1], 1ull);
        }
    } else if (level >= 0) {
        if (lane == 0 && !(ca.levels_used[c] & (1 << level))) atomicOr(&ca.levels_used[c], 1 << level);
        const unsigned mask = (unsigned)(ca.tab_off[c + 1] - tab - 1);
        const int ni = (int)(r[1] - r[0] + 1), nj = (int)(r[3] - r[2] + 1), nk = (int)(r[5] - r[4] + 1);
        fc.span[0] = ni;
        fc.span[1] = nj;
        fc.span[2] = nk;
        for (int q = lane; q < ni * nj * nk; q += FACE_LANES) {
            const long long i = r[0] + q % ni, j = r[2] + (q / ni) % nj, k = r[4] + q / (ni * nj);
            atomicAdd(&ca.counts[tab + (int)(cell_hash(i, j, k, level) & mask)], 1);
        }
    }
    if (lane == 0) ca.cells[f] = fc;
}

// Fill pass, warp per face over the faces the geometry pass visited (same
// list, same active chunks): the lanes split the face's stored cells and
// place the face in each cell's bucket range from k_grid_alloc, which
// returns every count to zero.
__global__ void k_contact_insert(ContactArrays ca, int c0, const uint32_t* __restrict__ face_list, long long n, Active act) {
    FOR_ACTIVE(act, n, 32, g) {
        int lane;
        const long long t = active_entity(act, g, 32, &lane);  // warp-uniform
        if (t >= n) continue;
        const long long f = face_list ? (long long)face_list[t] : ca.face_off[c0] + t;
        const int c = ca.face_contact[f];
        const int tab = ca.tab_off[c];
        if (ca.tab_off[c + 1] == tab) continue;
        const FaceCells fc = ca.cells[f];
        if (fc.level < 0 || fc.level >= GRID_LEVELS) continue;
        const int local = (int)(f - ca.face_off[c]);
        const unsigned mask = (unsigned)(ca.tab_off[c + 1] - tab - 1);
        const int ni = fc.span[0], nj = fc.span[1], nk = fc.span[2];
        for (int q = lane; q < ni * nj * nk; q += 32) {
            const long long i = fc.lo[0] + q % ni, j = fc.lo[1] + (q / ni) % nj, k = fc.lo[2] + q / (ni * nj);
            const int b = tab + (int)(cell_hash(i, j, k, fc.level) & mask);
            const int pos = atomicSub(&ca.counts[b], 1) - 1;
            ca.entries[ca.boff[b] + pos] = local;
        }
    }
}

__global__ void __launch_bounds__(FACE_TPB) k_contact_faces(ContactArrays ca, NodeArrays nd, Control* ctls, int c0,
                                                            const uint32_t* __restrict__ face_list, long long n, int run_mode, int do_grid,
                                                            Active act) {
    FOR_ACTIVE(act, n, FACE_LANES, g) {
        int lane;
        const long long t = active_entity(act, g, FACE_LANES, &lane);
        contact_face_body(ca, nd, ctls, c0, face_list, n, run_mode, do_grid, t, lane);
    }
}

// Thread per dynamic bucket: its range in the contact's entries, allocated
// with one atomic per warp (a warp's buckets belong to one table, since tables
// are multiples of 1024 buckets).
__global__ void k_grid_alloc(ContactArrays ca, int c0, int c1) {
    const long long b = (long long)ca.tab_off[c0] + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    if (b - lane >= ca.tab_off[c1]) return;  // warp-uniform
    // the warp's contact: the last c with tab_off[c] <= b (binary search)
    int lo = c0, hi = c1 - 1;
    const long long b0 = b - lane;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (ca.tab_off[mid] <= b0) lo = mid;
        else hi = mid - 1;
    }
    const int c = lo;
    const int cnt = ca.counts[b];
    int incl = cnt;
    for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += y;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    int base = 0;
    if (lane == 0 && total > 0) base = atomicAdd(&ca.ent_cursor[c], total);
    base = __shfl_sync(0xffffffffu, base, 0);
    ca.boff[b] = (unsigned)(ca.ent_off[c] + base + incl - cnt);
    ca.blen[b] = cnt;
}

// src/contact.rs:29-43
__device__ __forceinline__ bool point_in_triangle(const double* p, const double* a, const double* b, const double* c) {
    const double tol = 0.1;
    double v0[3], v1[3], v2[3];
    for (int d = 0; d < 3; ++d) {
        v0[d] = c[d] - a[d];
        v1[d] = b[d] - a[d];
        v2[d] = p[d] - a[d];
    }
    double d00 = v0[0] * v0[0] + v0[1] * v0[1] + v0[2] * v0[2];
    double d01 = v0[0] * v1[0] + v0[1] * v1[1] + v0[2] * v1[2];
    double d02 = v0[0] * v2[0] + v0[1] * v2[1] + v0[2] * v2[2];
    double d11 = v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2];
    double d12 = v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2];
    double inv = 1.0 / (d00 * d11 - d01 * d01);
    double uu = (d11 * d02 - d01 * d12) * inv;
    double vv = (d00 * d12 - d01 * d02) * inv;
    return uu >= -tol && vv >= -tol && uu + vv <= 1.0 + tol;
}

// The narrow test of one face for one point; returns the signed distance in *sd.
__device__ __forceinline__ bool face_hit(const FaceGeo& g, const double* p, double md, double* sd) {
    if (p[0] < g.lo[0] || p[0] > g.hi[0] || p[1] < g.lo[1] || p[1] > g.hi[1] || p[2] < g.lo[2] || p[2] > g.hi[2])
        return false;
    double dc0 = g.c[0] - p[0], dc1 = g.c[1] - p[1], dc2 = g.c[2] - p[2];
    double signed_d = -(g.n[0] * dc0 + g.n[1] * dc1 + g.n[2] * dc2);
    if (signed_d > 0.0 || signed_d < -md) return false;
    double proj[3] = {p[0] - g.n[0] * signed_d, p[1] - g.n[1] * signed_d, p[2] - g.n[2] * signed_d};
    bool inside = point_in_triangle(proj, g.x[0], g.x[1], g.x[2]) || point_in_triangle(proj, g.x[0], g.x[2], g.x[3]) ||
                  point_in_triangle(proj, g.x[1], g.x[2], g.x[3]) || point_in_triangle(proj, g.x[1], g.x[3], g.x[0]);
    *sd = signed_d;
    return inside;
}

// Block per big face (blocks stride over the search's list): every primary
// node of the face's contact inside the face's key box gets the narrow test,
// and a hit lowers the node's big_best to the face's local index, so
// big_best ends as the smallest big face that hits, whatever the order.
constexpr int BIG_TPB = 128;
constexpr int BIG_BLOCKS = 148 * 4;
__global__ void __launch_bounds__(BIG_TPB) k_contact_big(ContactArrays ca, NodeArrays nd) {
    __shared__ FaceGeo sg;
    __shared__ double sbox[6];
    const int count = min(*ca.big_count, (int)ca.big_cap);
    for (int k = blockIdx.x; k < count; k += gridDim.x) {  // block-uniform
        const long long f = ca.big_faces[k];
        __syncthreads();  // the previous face's readers are done
        if (threadIdx.x < sizeof(FaceGeo) / sizeof(double))
            reinterpret_cast<double*>(&sg)[threadIdx.x] = reinterpret_cast<const double*>(ca.geo + f)[threadIdx.x];
        if (threadIdx.x < 6) sbox[threadIdx.x] = ca.big_box[6 * (long long)k + threadIdx.x];
        __syncthreads();
        const int c = ca.face_contact[f];
        const int local = (int)(f - ca.face_off[c]);
        const double md = ca.max_distance[c];
        const long long s1 = ca.slave_off[c + 1];
        for (long long s = ca.slave_off[c] + threadIdx.x; s < s1; s += BIG_TPB) {
            const long long n = ca.slaves[s];
            const double p[3] = {nd.pos[3 * n] + nd.u[3 * n], nd.pos[3 * n + 1] + nd.u[3 * n + 1], nd.pos[3 * n + 2] + nd.u[3 * n + 2]};
            if (!(p[0] >= sbox[0] && p[0] <= sbox[3] && p[1] >= sbox[1] && p[1] <= sbox[4] && p[2] >= sbox[2] && p[2] <= sbox[5])) continue;
            double sd;
            if (face_hit(sg, p, md, &sd)) atomicMin(&ca.big_best[s], local);
        }
    }
}

// One reaction event of a hit: key 2s (the primary node's own +F) or 2s+1
// (-F/4 on a node of the hit face) appended to the contact node's list, or
// to the shared pool once the list holds EV_CAP; fixed nodes take none when
// the pass skips them.
__device__ __forceinline__ void emit_event(const ContactArrays& ca, uint32_t code, uint32_t key, int skip_fixed) {
    if (skip_fixed && (code & CN_FIXED)) return;
    const uint32_t cn = code & ~CN_FIXED;
    const int slot = atomicAdd(&ca.ev_count[cn], 1);
    if (slot < EV_CAP) {
        ca.ev_list[(long long)cn * EV_CAP + slot] = key;
    } else {
        if (slot == EV_CAP) ca.gather_work[atomicAdd(ca.gather_count, 1)] = (int)cn;  // the node turns heavy, once
        const int p = atomicAdd(ca.ev_pool_n, 1);
        if (p < ca.ev_pool_cap) ca.ev_pool[p] = make_uint2(cn, key);
    }
}

// The penalty force of primary-node entry s (node n of contact c) on its
// first-hit face `best` (src/contact.rs:130-153: depth capped at 0.1 md,
// stiffness limited to 0.1 m / dt^2, force capped at m * 1e5), and its five
// reaction events: +F on the node, -F/4 on each of the face's four corners
// (a node on two corners takes two). FORCE_LANES lanes share an entry: lane
// j emits corner j's event, lane 0 also the node's own and the force.
constexpr int FORCE_LANES = 4;
__device__ __forceinline__ void record_hit(const ContactArrays& ca, long long s, int c, long long n, int best, double best_sd, double dt,
                                           const double* __restrict__ masses, const FaceGeo& g, int skip_fixed, int lane) {
    const long long F = ca.face_off[c] + best;
    const uint32_t key = 2u * (uint32_t)s;
    emit_event(ca, ca.face_cn[4 * F + lane], key + 1u, skip_fixed);
    if (lane != 0) return;
    emit_event(ca, ca.slave_cn[s], key, skip_fixed);
    const double md = ca.max_distance[c];
    const double m = masses[n];
    const double depth = fmin(-best_sd, 0.1 * md);
    const double k_pen = fmin(ca.stiffness[c] * ca.slave_scale[s], 0.1 * m / (dt * dt));
    const double mag = fmin(k_pen * depth, m * 1.0e5);
    ca.hit[s] = best;
    ca.hit_force[3 * s] = mag * g.n[0];
    ca.hit_force[3 * s + 1] = mag * g.n[1];
    ca.hit_force[3 * s + 2] = mag * g.n[2];
    atomicAdd(&ca.pen_count[c], 1ull);
    // + 0.0 turns a zero depth's -0.0 (signed_d == +0.0 hits) into +0.0, whose
    // bits order below every positive depth.
    atomicMax(&ca.pen_max_bits[c], (unsigned long long)__double_as_longlong(-best_sd + 0.0));
}

// First-hit search: LANES lanes per primary node (a power of two <= 32,
// chosen per context by the launch autotuner) test the faces its broad phase
// offers — the static grid's bucket, or the dynamic grid's bucket at every
// level in use, starting from the smallest big face that hit — or every face
// of the contact when it has no grid (small contacts), or this is a drop-in
// call on a static contact; and keep the smallest face index that hits: the
// face the reference's in-order scan with `break` finds
// (src/contact.rs:115-157). Lane 0 sets the node's big_best back to
// BIG_NONE for the next search, also when its crash has stopped.
template <int LANES>
__device__ __forceinline__ void contact_slave_body(const ContactArrays& ca, const NodeArrays& nd, const Control* ctls, int c0, int c1,
                                                   int run_mode, double dt_override, const double* __restrict__ masses, long long s,
                                                   bool live, int lane) {
    const Control* ctl = nullptr;
    bool reset_big = false;
    if (live) {
        const int c = ca.slave_contact[s];
        reset_big = lane == 0 && ca.tab_off[c + 1] > ca.tab_off[c] && !ca.exhaustive;
        ctl = ctls + ca.contact_slot[c];
        if (run_mode && ctl->done) live = false;
    }
    int best = INT_MAX;
    double best_sd = 0.0, sd;
    int c = 0;
    long long n = 0;
    double p[3] = {0.0, 0.0, 0.0}, md = 0.0;
    const FaceGeo* geo = nullptr;
    if (live) {
        c = ca.slave_contact[s];
        n = ca.slaves[s];
        p[0] = nd.pos[3 * n] + nd.u[3 * n];
        p[1] = nd.pos[3 * n + 1] + nd.u[3 * n + 1];
        p[2] = nd.pos[3 * n + 2] + nd.u[3 * n + 2];
        md = ca.max_distance[c];
        const long long fb = ca.face_off[c];
        const int nf = (int)(ca.face_off[c + 1] - fb);
        geo = ca.geo + fb;
        const long long st0 = ca.st_tab_off[c], st1 = ca.st_tab_off[c + 1];
        const int tab = ca.tab_off[c];
        const bool dyn_grid = ca.tab_off[c + 1] > tab;
        bool all = false;
        const double* box = ca.st_box + 6 * c;
        if (run_mode && st1 > st0 && !ca.exhaustive &&
            !(p[0] >= box[0] && p[0] <= box[3] && p[1] >= box[1] && p[1] <= box[4] && p[2] >= box[2] && p[2] <= box[5])) {
            // Outside every key box of the fixed faces: nothing to test.
        } else if (run_mode && st1 > st0 && !ca.exhaustive) {
            // Static grid: the bucket of the point's cell, exact.
            const unsigned mask = (unsigned)(st1 - st0 - 1);
            const long long bk = st0 + (point_cell_hash(p, ca.cell[c], 0) & mask);
            const uint32_t e0 = ca.st_off[bk + c], e1 = ca.st_off[bk + c + 1];
            for (uint32_t k = e0 + lane; k < e1; k += LANES) {
                const int f = ca.st_entries[k];
                if (f < best && face_hit(geo[f], p, md, &sd)) { best = f; best_sd = sd; }
            }
        } else if (dyn_grid && !ca.exhaustive) {
            const int big = ca.big_best[s];
            if (big != BIG_NONE && face_hit(geo[big], p, md, &sd)) {  // always hits: the big-face pass's own test
                best = big;
                best_sd = sd;
            }
            const unsigned mask = (unsigned)(ca.tab_off[c + 1] - tab - 1);
            const int used = ca.levels_used[c];
            static_assert(GRID_LEVELS == 2, "the lane split below assumes two grid levels");
            if (LANES >= 2 && used == 3) {
                // both levels in use: half the lanes scan each, concurrently
                const int level = lane < LANES / 2 ? 0 : 1;
                const double cs = level ? ca.cell[c] * 4.0 : ca.cell[c];
                const int b = tab + (int)(point_cell_hash(p, cs, level) & mask);
                const unsigned e0 = ca.boff[b];
                const int cnt = ca.blen[b];
                for (int k = lane % (LANES / 2); k < cnt; k += LANES / 2) {
                    const int f = ca.entries[e0 + k];
                    if (f < best && face_hit(geo[f], p, md, &sd)) { best = f; best_sd = sd; }
                }
            } else {
                double cs = ca.cell[c];
                for (int level = 0; level < GRID_LEVELS; ++level, cs *= 4.0) {
                    if (!(used & (1 << level))) continue;
                    const int b = tab + (int)(point_cell_hash(p, cs, level) & mask);
                    const unsigned e0 = ca.boff[b];
                    const int cnt = ca.blen[b];
                    for (int k = lane; k < cnt; k += LANES) {
                        const int f = ca.entries[e0 + k];
                        if (f < best && face_hit(geo[f], p, md, &sd)) { best = f; best_sd = sd; }
                    }
                }
            }
        } else {
            all = true;
        }
        if (all)
            for (int f = lane; f < nf; f += LANES)
                if (f < best && face_hit(geo[f], p, md, &sd)) { best = f; best_sd = sd; }
    }
#pragma unroll
    for (int off = LANES / 2; off > 0; off >>= 1) {
        const int ob = __shfl_down_sync(0xffffffffu, best, off, LANES);
        const double osd = __shfl_down_sync(0xffffffffu, best_sd, off, LANES);
        if (ob < best) { best = ob; best_sd = osd; }
    }
    if (reset_big) ca.big_best[s] = BIG_NONE;
    if (!live || lane != 0) return;
    if (best == INT_MAX) {
        ca.hit[s] = -1;
        return;
    }
    ca.hit[s] = best;
    ca.hit_sd[s] = best_sd;
}

// run: the entries of `list` (grid_slaves or st_slaves, over their active
// chunks), else the entries of contacts [c0, c1).
template <int LANES>
__global__ void k_contact_slaves(ContactArrays ca, NodeArrays nd, Control* ctls, int c0, int c1, int run_mode, double dt_override,
                                 const double* __restrict__ masses, long long n_slaves, const uint32_t* __restrict__ list, Active act) {
    const long long s_begin = ca.slave_off[c0];
    FOR_ACTIVE(act, n_slaves, LANES, g) {
        int lane;
        const long long e = active_entity(act, g, LANES, &lane);
        const bool live = e < n_slaves;
        const long long s = !live ? 0 : (list ? (long long)list[e] : s_begin + e);
        contact_slave_body<LANES>(ca, nd, ctls, c0, c1, run_mode, dt_override, masses, s, live, lane);
    }
}

constexpr int ST_LANES = 2;  // lanes per entry of a static-grid contact (a box test, then a short bucket)

// Contacts searched exhaustively (fewer faces than the grid threshold), a
// few blocks per contact (gridDim.y, brute_split) sharing its primary-node
// entries: each block stages the contact's face geometry in shared memory
// and each thread scans the faces in order for one primary node and stops at
// the first hit, as src/contact.rs:115-157 does.
constexpr int BRUTE_TPB = 128;
constexpr int BRUTE_MAX_FACES = 255;  // 255 x 192 B fits the default 48 KB of shared memory
template <int BRUTE_LANES>
__global__ void __launch_bounds__(BRUTE_TPB) k_contact_brute(ContactArrays ca, NodeArrays nd, Control* ctls, const int* __restrict__ list,
                                                            int single, int run_mode, double dt_override, const double* __restrict__ masses) {
    extern __shared__ double sbuf[];
    FaceGeo* sgeo = reinterpret_cast<FaceGeo*>(sbuf);
    const int c = list ? list[blockIdx.x] : single;
    const Control* ctl = ctls + ca.contact_slot[c];
    if (run_mode && ctl->done) return;  // block-uniform
    const long long fb = ca.face_off[c];
    const int nf = (int)(ca.face_off[c + 1] - fb);
    const double* src = reinterpret_cast<const double*>(ca.geo + fb);
    for (int k = threadIdx.x; k < nf * (int)(sizeof(FaceGeo) / sizeof(double)); k += blockDim.x) sbuf[k] = src[k];
    __syncthreads();
    const double md = ca.max_distance[c];
    // BRUTE_LANES lanes per primary node, each scanning every BRUTE_LANES-th
    // face in order up to its first hit; the smallest hit index wins.
    const int lane = threadIdx.x % BRUTE_LANES;
    const long long s_end = ca.slave_off[c + 1];
    // the contact's entries are shared by gridDim.y blocks, in turns of a block's worth
    const long long per_block = blockDim.x / BRUTE_LANES;
    for (long long base = ca.slave_off[c] + blockIdx.y * per_block; base < s_end; base += gridDim.y * per_block) {  // block-uniform
        const long long s = base + threadIdx.x / BRUTE_LANES;
        const bool live = s < s_end;
        long long n = 0;
        int best = INT_MAX;
        double best_sd = 0.0, sd;
        if (live) {
            n = ca.slaves[s];
            const double p[3] = {nd.pos[3 * n] + nd.u[3 * n], nd.pos[3 * n + 1] + nd.u[3 * n + 1], nd.pos[3 * n + 2] + nd.u[3 * n + 2]};
            for (int f = lane; f < nf; f += BRUTE_LANES)
                if (face_hit(sgeo[f], p, md, &sd)) {
                    best = f;
                    best_sd = sd;
                    break;
                }
        }
#pragma unroll
        for (int off = BRUTE_LANES / 2; off > 0; off >>= 1) {
            const int ob = __shfl_down_sync(0xffffffffu, best, off, BRUTE_LANES);
            const double osd = __shfl_down_sync(0xffffffffu, best_sd, off, BRUTE_LANES);
            if (ob < best) {
                best = ob;
                best_sd = osd;
            }
        }
        if (!live || lane != 0) continue;
        if (best == INT_MAX) {
            ca.hit[s] = -1;
            continue;
        }
        ca.hit[s] = best;
        ca.hit_sd[s] = best_sd;
    }
}

// The penalty forces of the hits the search found (src/contact.rs:130-153),
// thread per primary-node entry: run the search finished before (possibly
// overlapping other work); this pass needs the step's dt and records the
// reaction events and the penetration counters.
__global__ void k_contact_force(ContactArrays ca, Control* ctls, int c0, int run_mode, double dt_override,
                                const double* __restrict__ masses, long long n_slaves, int skip_fixed, int next_step) {
    const Active act = run_mode ? ca.act_allslave : Active{nullptr, nullptr};
    const long long s0 = ca.slave_off[c0];
    FOR_ACTIVE(act, n_slaves, FORCE_LANES, g) {
        int lane;
        const long long e = active_entity(act, g, FORCE_LANES, &lane);
        if (e >= n_slaves) continue;
        const long long s = s0 + e;
        const int best = ca.hit[s];
        if (best < 0) continue;
        const int c = ca.slave_contact[s];
        const Control* ctl = ctls + ca.contact_slot[c];
        if (run_mode && ctl->done) continue;
        const double dt = dt_override > 0.0 ? dt_override : (next_step ? next_step_dt(ctl) : step_dt(ctl));
        record_hit(ca, s, c, ca.slaves[s], best, ca.hit_sd[s], dt, masses,
                   ca.geo[ca.face_off[c] + best], skip_fixed, lane);
    }
}

// End of a force pass, one block, once both gathers are done: the pass's
// heavy nodes (those listed in gather_work) get their event counts back to
// zero, then the pool and the heavy list are emptied, so every pass starts
// from zero counts. The heavy gather cannot clear its own nodes' counts: the
// other gather, beside it on a second stream or after it on the same
// stream, reads them to skip those nodes.
constexpr int RESET_TPB = 512;
__global__ void __launch_bounds__(RESET_TPB) k_contact_reset(ContactArrays ca) {
    const int count = *ca.gather_count;
    for (int w = threadIdx.x; w < count; w += RESET_TPB) ca.ev_count[ca.gather_work[w]] = 0;
    __syncthreads();  // every thread has read the count
    if (threadIdx.x == 0) {
        *ca.ev_pool_n = 0;
        *ca.gather_count = 0;
    }
}

constexpr int GATHER_TPB = 128;
constexpr int HEAVY_TPB = 256;
constexpr int HEAVY_KEYS = 2048;     // events a block sorts itself
constexpr int WALK_PER_THREAD = 4;   // consecutive primary nodes per thread in a walk round
constexpr int HEAVY_BLOCKS = 296;    // 2 x 148 SMs
// keys of one walk round: up to 5 per entry (own + four corners)
constexpr int HEAVY_BUF = HEAVY_TPB * WALK_PER_THREAD * 5 > HEAVY_KEYS ? HEAVY_TPB * WALK_PER_THREAD * 5 : HEAVY_KEYS;

// Adds one event to (sx, sy, sz) the way src/contact.rs:146-153 adds it to
// f_ext: += F for the primary node itself, -= 0.25 F for a face corner.
__device__ __forceinline__ void apply_event(bool face, double fx, double fy, double fz, double& sx, double& sy, double& sz) {
    if (face) {
        sx -= 0.25 * fx;
        sy -= 0.25 * fy;
        sz -= 0.25 * fz;
    } else {
        sx += fx;
        sy += fy;
        sz += fz;
    }
}

// Ordered reaction gather, one thread per contact node. The node's events
// carry keys 2s (own) and 2s+1 (face) of the global primary-node index s;
// contacts are numbered in order and so are their entries, so ascending keys
// are the order in which src/contact.rs:146-153 adds the reactions to f_ext,
// contact after contact. Up to EV_CAP keys are sorted in registers (a
// bitonic network) and their forces loaded together; a node with more goes
// to k_contact_gather_heavy (the force pass listed it), which writes its
// output; its count stays until k_contact_reset at the next pass, so this
// gather skips it whichever kernel runs first. The gather zeroes the other
// nodes' event counts for the next pass. In a run it also writes the node's
// half-step u to u_next (fixed nodes and stopped crashes keep theirs), so
// the next step's search can start before the half step.
__device__ __forceinline__ void gather_body(const ContactArrays& ca, const NodeArrays& nd, const Control* ctls, int c0, int c1,
                                            int run_mode, double* __restrict__ f_out, int skip_fixed, long long i) {
    if (i >= ca.n_cnodes) return;
    const long long n = ca.cnode[i];
    if ((skip_fixed && nd.fixed[n]) || (run_mode && ctls[nd.node_slot[n]].done)) return;
    if (!run_mode) {  // a drop-in call writes the nodes with a role in contacts [c0, c1)
        bool touched = false;
        for (uint32_t r = ca.cnode_off[i]; r < ca.cnode_off[i + 1]; ++r) {
            const int c = ca.crole_contact[r];
            touched |= c >= c0 && c < c1;
        }
        if (!touched) return;
    }
    const int cnt = ca.ev_count[i];
    if (cnt > EV_CAP) return;  // k_contact_gather_heavy's node
    double sx = 0.0, sy = 0.0, sz = 0.0;
    if (cnt > 0) {
        ca.ev_count[i] = 0;
        uint32_t k[EV_CAP];
        const uint4* row = reinterpret_cast<const uint4*>(ca.ev_list + i * EV_CAP);
#pragma unroll
        for (int q = 0; q < EV_CAP / 4; ++q) {
            const uint4 v = row[q];
            k[4 * q] = v.x;
            k[4 * q + 1] = v.y;
            k[4 * q + 2] = v.z;
            k[4 * q + 3] = v.w;
        }
#pragma unroll
        for (int j = 0; j < EV_CAP; ++j)
            if (j >= cnt) k[j] = 0xFFFFFFFFu;
#pragma unroll
        for (int size = 2; size <= EV_CAP; size <<= 1)
#pragma unroll
            for (int stride = size >> 1; stride > 0; stride >>= 1)
#pragma unroll
                for (int a = 0; a < EV_CAP; ++a) {
                    const int b = a ^ stride;
                    if (b > a) {
                        const uint32_t lo = min(k[a], k[b]), hi = max(k[a], k[b]);
                        const bool up = (a & size) == 0;
                        k[a] = up ? lo : hi;
                        k[b] = up ? hi : lo;
                    }
                }
#pragma unroll
        for (int g = 0; g < EV_CAP; g += 8) {
            if (g < cnt) {
                double fx[8], fy[8], fz[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const long long e = (long long)(k[g + j] >> 1);
                    const bool ok = g + j < cnt;
                    fx[j] = ok ? __ldg(ca.hit_force + 3 * e) : 0.0;
                    fy[j] = ok ? __ldg(ca.hit_force + 3 * e + 1) : 0.0;
                    fz[j] = ok ? __ldg(ca.hit_force + 3 * e + 2) : 0.0;
                }
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    if (g + j < cnt) apply_event(k[g + j] & 1u, fx[j], fy[j], fz[j], sx, sy, sz);
            }
        }
    }
    f_out[3 * n] = sx;
    f_out[3 * n + 1] = sy;
    f_out[3 * n + 2] = sz;
}

__global__ void __launch_bounds__(GATHER_TPB) k_contact_gather(ContactArrays ca, NodeArrays nd, Control* ctls, int c0, int c1,
                                                               int run_mode, double* __restrict__ f_out, int skip_fixed) {
    const Active act = run_mode ? ca.act_cnode : Active{nullptr, nullptr};
    FOR_ACTIVE(act, ca.n_cnodes, 1, g) {
        int lane;
        gather_body(ca, nd, ctls, c0, c1, run_mode, f_out, skip_fixed, active_entity(act, g, 1, &lane));
    }
}

// Threads 0, 1 and 2 add, in order, component 0, 1 and 2 of the events
// listed in keys[0, count) (ascending) to their running sum acc, the
// forces fetched HEAVY_TPB at a time by the whole block. The components'
// sums are independent, so each is the reference's sequence for its axis.
__device__ void heavy_sum(const ContactArrays& ca, const uint32_t* keys, int count, double (*sf)[3], double& acc) {
    for (int b0 = 0; b0 < count; b0 += HEAVY_TPB) {  // block-uniform
        const int t = b0 + threadIdx.x;
        if (t < count) {
            const long long e = (long long)(keys[t] >> 1);
            sf[threadIdx.x][0] = ca.hit_force[3 * e];
            sf[threadIdx.x][1] = ca.hit_force[3 * e + 1];
            sf[threadIdx.x][2] = ca.hit_force[3 * e + 2];
        }
        __syncthreads();
        if (threadIdx.x < 3) {
            const int m = min(HEAVY_TPB, count - b0);
            const int d = threadIdx.x;
            double a = acc;
#pragma unroll 4
            for (int j = 0; j < m; ++j) {
                const double fd = sf[j][d];
                if (keys[b0 + j] & 1u) a -= 0.25 * fd;
                else a += fd;
            }
            acc = a;
        }
        __syncthreads();
    }
}

// The events of contact node i (node n) rebuilt without its lists: the block
// walks, contact after contact (its roles are grouped by contact, in order),
// the contact's primary nodes in rounds of HEAVY_TPB x WALK_PER_THREAD
// consecutive entries; per entry an own hit (one of the node's entries in
// the contact) gives key 2s and each corner of the hit face that is n gives
// 2s+1. A block scan places the round's keys in entry order (already
// ascending) and heavy_sum adds them.
__device__ void walk_node(const ContactArrays& ca, int c0, int c1, long long i, long long n, uint32_t* keys, double (*sf)[3],
                          int* s_warp, double& acc) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t r_end = ca.cnode_off[i + 1];
    for (uint32_t r = ca.cnode_off[i], r1; r < r_end; r = r1) {
        const int c = ca.crole_contact[r];
        r1 = r + 1;
        while (r1 < r_end && ca.crole_contact[r1] == c) ++r1;
        if (c < c0 || c >= c1) continue;
        if (threadIdx.x == 0) atomicAdd(&ca.search_stats[3 * c + 2], 1ull);
        const long long sb = ca.slave_off[c], se = ca.slave_off[c + 1];
        const uint32_t* faces = ca.faces + 4 * ca.face_off[c];
        for (long long base = sb; base < se; base += HEAVY_TPB * WALK_PER_THREAD) {  // block-uniform
            int own_j[WALK_PER_THREAD], m_j[WALK_PER_THREAD];
            int mine = 0;
#pragma unroll
            for (int j = 0; j < WALK_PER_THREAD; ++j) {
                const long long s = base + threadIdx.x * WALK_PER_THREAD + j;
                own_j[j] = 0;
                m_j[j] = 0;
                if (s < se) {
                    const int h = ca.hit[s];
                    if (h >= 0) {
                        const uint32_t* qn = faces + 4 * (long long)h;
                        for (uint32_t q = r; q < r1; ++q) own_j[j] |= ca.crole_slave[q] == s - sb ? 1 : 0;
                        m_j[j] = (qn[0] == n ? 1 : 0) + (qn[1] == n ? 1 : 0) + (qn[2] == n ? 1 : 0) + (qn[3] == n ? 1 : 0);
                    }
                }
                mine += own_j[j] + m_j[j];
            }
            int incl = mine;  // block exclusive scan of the keys per thread
            for (int off = 1; off < 32; off <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, off);
                if (lane >= off) incl += y;
            }
            if (lane == 31) s_warp[warp] = incl;
            __syncthreads();
            int before = 0, total = 0;
            for (int k = 0; k < HEAVY_TPB / 32; ++k) {
                const int v = s_warp[k];
                before += k < warp ? v : 0;
                total += v;
            }
            int pos = before + incl - mine;
#pragma unroll
            for (int j = 0; j < WALK_PER_THREAD; ++j) {
                const uint32_t key = 2u * (uint32_t)(base + threadIdx.x * WALK_PER_THREAD + j);
                if (own_j[j]) keys[pos++] = key;
                for (int a = 0; a < m_j[j]; ++a) keys[pos++] = key + 1u;
            }
            __syncthreads();
            heavy_sum(ca, keys, total, sf, acc);  // ends with a barrier: keys and s_warp are free again
        }
    }
}

// Contact nodes with more than EV_CAP events, a block each (blocks stride
// over the list): the node's list and its events in the shared pool are
// collected (EV_CAP + pool = the count when nothing was dropped), sorted by a
// bitonic sort in shared memory and added in order. A node whose events do
// not fit HEAVY_KEYS, or lost some to a full pool, is rebuilt by walk_node.
// The nodes' event counts are left for k_contact_reset.
__global__ void __launch_bounds__(HEAVY_TPB) k_contact_gather_heavy(ContactArrays ca, NodeArrays nd, const Control* ctls, int c0, int c1,
                                                                    int run_mode, double* __restrict__ f_out) {
    __shared__ uint32_t keys[HEAVY_BUF];
    __shared__ double sf[HEAVY_TPB][3];
    __shared__ int s_warp[HEAVY_TPB / 32];
    __shared__ int s_n;
    const int count = *ca.gather_count;
    for (int w = blockIdx.x; w < count; w += gridDim.x) {  // block-uniform
        const long long i = ca.gather_work[w];
        const int cnt = ca.ev_count[i];  // final: the force pass is done
        const long long n = ca.cnode[i];
        double acc = 0.0;  // thread d < 3: component d of the running sum
        bool walk = cnt > HEAVY_KEYS;
        if (!walk) {
            if (threadIdx.x == 0) s_n = 0;
            __syncthreads();
            for (int t = threadIdx.x; t < EV_CAP; t += HEAVY_TPB) keys[t] = ca.ev_list[i * EV_CAP + t];
            const int np = (int)min((long long)*ca.ev_pool_n, ca.ev_pool_cap);
            for (int p = threadIdx.x; p < np; p += HEAVY_TPB) {
                const uint2 e = ca.ev_pool[p];
                if (e.x == (uint32_t)i) {
                    const int q = EV_CAP + atomicAdd(&s_n, 1);
                    if (q < HEAVY_KEYS) keys[q] = e.y;
                }
            }
            __syncthreads();
            walk = EV_CAP + s_n != cnt;  // block-uniform
        }
        if (walk) {
            __syncthreads();
            walk_node(ca, c0, c1, i, n, keys, sf, s_warp, acc);
        } else {
            int P = EV_CAP;
            while (P < cnt) P <<= 1;
            for (int t = cnt + threadIdx.x; t < P; t += HEAVY_TPB) keys[t] = 0xFFFFFFFFu;
            __syncthreads();
            for (int size = 2; size <= P; size <<= 1)
                for (int stride = size >> 1; stride > 0; stride >>= 1) {
                    for (int a = threadIdx.x; a < P; a += HEAVY_TPB) {
                        const int b = a ^ stride;
                        if (b > a) {
                            const uint32_t x = keys[a], y = keys[b];
                            const bool up = (a & size) == 0;
                            if ((x > y) == up) {
                                keys[a] = y;
                                keys[b] = x;
                            }
                        }
                    }
                    __syncthreads();
                }
            heavy_sum(ca, keys, cnt, sf, acc);
        }
        if (threadIdx.x < 3) {
            f_out[3 * n + threadIdx.x] = acc;
        }
        __syncthreads();  // every thread is done with s_n and the shared buffers
    }
}

// ---------------------------------------------------------------------------
// FP64 vehicle reductions (delta-v, crush, separation rule), one block per
// vehicle (or per vehicle slice), fixed summation order.
// ---------------------------------------------------------------------------
constexpr int VEH_TPB = 256;

__global__ void __launch_bounds__(VEH_TPB) k_vehicle_sums(VehicleArrays va, const double* __restrict__ mass, const double* __restrict__ v,
                                                          const double* __restrict__ v0, double* __restrict__ out) {
    __shared__ double s[7][VEH_TPB];
    const int veh = blockIdx.x;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    for (long long i = va.off[veh] + threadIdx.x; i < va.off[veh + 1]; i += VEH_TPB) {
        const long long n = va.nodes[i];
        const double m = mass[n];
        acc[0] += m;
        for (int d = 0; d < 3; ++d) {
            acc[1 + d] += m * v[3 * n + d];
            acc[4 + d] += m * v0[3 * n + d];
        }
    }
    for (int k = 0; k < 7; ++k) s[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int w = VEH_TPB / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 7; ++k) s[k][threadIdx.x] += s[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 7; ++k) out[7 * veh + k] = s[k][0];
}

// u_x of listed nodes (the crush measure's inputs).
__global__ void k_gather_ux(long long n, const uint32_t* __restrict__ nodes, const double* __restrict__ u, double* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = u[3 * (long long)nodes[i]];
}

// Blocks a vehicle's separation-rule reduction uses: one per 2048 nodes, at
// most VX_BLOCKS. It depends only on the vehicle itself, so a crash reduces
// in the same order alone and inside a batch.
__device__ __forceinline__ long long vx_blocks_of(long long len) {
    const long long b = (len + 2047) / 2048;
    return b < 1 ? 1 : (b > VX_BLOCKS ? VX_BLOCKS : b);
}

// Mean x-velocity partial sums for the separation rule: vx_blocks_of(len)
// blocks per vehicle, each over a contiguous slice of the vehicle's nodes
// (the launch has va.vx_blocks, the largest count; surplus blocks write zero
// partials); k_step_end adds the partials in block order.
__global__ void __launch_bounds__(VEH_TPB) k_vehicle_vx(VehicleArrays va, const double* __restrict__ mass, const double* __restrict__ v,
                                                        Control* ctls) {
    __shared__ double sm[VEH_TPB], sp[VEH_TPB];
    const int veh = blockIdx.x / va.vx_blocks, b = blockIdx.x % va.vx_blocks;
    Control* ctl = ctls + va.slot[veh];
    const int lv = va.local[veh];
    if (ctl->done || lv >= 4) return;
    const long long n0 = va.off[veh], len = va.off[veh + 1] - va.off[veh];
    const long long nb = vx_blocks_of(len);
    const long long per = (len + nb - 1) / nb;
    const long long lo = b < nb ? n0 + b * per : n0 + len, hi = min(lo + per, n0 + len);
    double m_acc = 0.0, p_acc = 0.0;
    for (long long i = lo + threadIdx.x; i < hi; i += VEH_TPB) {
        const long long n = va.nodes[i];
        m_acc += mass[n];
        p_acc += mass[n] * v[3 * n];
    }
    sm[threadIdx.x] = m_acc;
    sp[threadIdx.x] = p_acc;
    __syncthreads();
    for (int w = VEH_TPB / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            sm[threadIdx.x] += sm[threadIdx.x + w];
            sp[threadIdx.x] += sp[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        ctl->vx_part[lv][b][0] = sm[0];
        ctl->vx_part[lv][b][1] = sp[0];
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
void launch_setup_geometry(cudaStream_t s, long long e_begin, long long n_all, const double* pos, const uint32_t* conn_all,
                           const int32_t* part, const double* mat, const int64_t* hc_index, const uint32_t* elem_slot, long long stride,
                           float4* planes, double* volume, double* lumped, double* dt_factor, double* elem_mass, int* bad,
                           const int64_t* sc_index, long long n_sc, double* sc_geo) {
    if (n_all <= e_begin) return;
    k_setup_geometry8<<<(unsigned)blocks_for(n_all - e_begin, GEO_PER_BLOCK), GEO_TPB, 0, s>>>(
        e_begin, n_all, pos, conn_all, part, mat, hc_index, elem_slot, stride, planes, volume, lumped, dt_factor, elem_mass, bad, sc_index,
        n_sc, sc_geo);
}
void launch_node_masses(cudaStream_t s, long long n, const uint32_t* off, const uint32_t* slot, const double* lumped,
                        double* mass, double* inv_mass) {
    k_node_masses<<<(unsigned)blocks_for(n, TPB), TPB, 0, s>>>(n, off, slot, lumped, mass, inv_mass);
}
// Scratch of launch_incidence: sort keys and values, their second buffers,
// three count arrays, three offset arrays and CUB's temporary storage.
struct IncidenceScratch {
    size_t keys, keys2, vals, vals2, cnt, rel, temp, total;
};
IncidenceScratch incidence_layout(long long ne, long long nn) {
    const size_t m = 8 * (size_t)std::max<long long>(ne, 1), c = (size_t)nn + 1;
    size_t sort_bytes = 0, scan_bytes = 0;
    cub::DoubleBuffer<uint32_t> k(nullptr, nullptr), v(nullptr, nullptr);
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, k, v, (int)m, 0, 32);
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (uint32_t*)nullptr, (uint32_t*)nullptr, (int)c);
    auto up = [](size_t b) { return (b + 255) / 256 * 256; };
    IncidenceScratch l;
    l.keys = 0;
    l.keys2 = l.keys + up(4 * m);
    l.vals = l.keys2 + up(4 * m);
    l.vals2 = l.vals + up(4 * m);
    l.cnt = l.vals2 + up(4 * m);
    l.rel = l.cnt + 3 * up(4 * c);
    l.temp = l.rel + 3 * up(4 * c);
    l.total = l.temp + up(std::max(sort_bytes, scan_bytes));
    return l;
}
size_t incidence_scratch_bytes(long long ne, long long nn) { return incidence_layout(ne, nn).total; }

int launch_incidence(cudaStream_t s, long long e0, long long ne, long long n0, long long nn, const uint32_t* conn_all,
                     const int64_t* hc_index, const int64_t* sc_index, uint32_t base_all, uint32_t base_hc, uint32_t base_sc,
                     uint32_t* all_off, uint32_t* all_slot, uint32_t* hc_off, uint32_t* hc_slot, uint32_t* sc_off, uint32_t* sc_slot,
                     uint32_t* hc_ell, void* scratch) {
    if (nn <= 0) return 0;
    const IncidenceScratch l = incidence_layout(ne, nn);
    char* b = static_cast<char*>(scratch);
    const size_t m = 8 * (size_t)ne, c = (size_t)nn + 1;
    auto up = [](size_t x) { return (x + 255) / 256 * 256; };
    uint32_t* keys = reinterpret_cast<uint32_t*>(b + l.keys);
    uint32_t* keys2 = reinterpret_cast<uint32_t*>(b + l.keys2);
    uint32_t* vals = reinterpret_cast<uint32_t*>(b + l.vals);
    uint32_t* vals2 = reinterpret_cast<uint32_t*>(b + l.vals2);
    uint32_t* cnt[3];
    uint32_t* rel[3];
    for (int k = 0; k < 3; ++k) {
        cnt[k] = reinterpret_cast<uint32_t*>(b + l.cnt + k * up(4 * c));
        rel[k] = reinterpret_cast<uint32_t*>(b + l.rel + k * up(4 * c));
    }
    void* temp = b + l.temp;
    const size_t temp_bytes = l.total - l.temp;
    for (int k = 0; k < 3; ++k)
        if (cudaMemsetAsync(cnt[k], 0, 4 * c, s) != cudaSuccess) return -1;
    if (ne > 0)
        k_incidence_count<<<(unsigned)blocks_for(ne, TPB), TPB, 0, s>>>(e0, ne, n0, conn_all, hc_index, keys, vals, cnt[0], cnt[1], cnt[2]);
    for (int k = 0; k < 3; ++k) {
        size_t tb = temp_bytes;
        if (cub::DeviceScan::ExclusiveSum(temp, tb, cnt[k], rel[k], (int)c, s) != cudaSuccess) return -1;
    }
    if (m > 0) {
        int bits = 1;
        while (bits < 32 && ((uint64_t)1 << bits) < (uint64_t)nn) ++bits;
        cub::DoubleBuffer<uint32_t> dk(keys, keys2), dv(vals, vals2);
        size_t tb = temp_bytes;
        if (cub::DeviceRadixSort::SortPairs(temp, tb, dk, dv, (int)m, 0, bits, s) != cudaSuccess) return -1;
        if (cudaMemcpyAsync(all_slot + base_all, dv.Current(), 4 * m, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return -1;
    }
    k_incidence_split<<<(unsigned)blocks_for(nn + 1, TPB), TPB, 0, s>>>(nn, rel[0], rel[1], rel[2], base_all, base_hc, base_sc, hc_index,
                                                                     sc_index, all_slot, all_off, hc_off, hc_slot, sc_off, sc_slot, hc_ell);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
void launch_init_state(cudaStream_t s, long long h_begin, long long n_hc, long long stride, float4* state) {
    if (n_hc <= h_begin) return;
    k_init_state<<<(unsigned)blocks_for(n_hc - h_begin, TPB), TPB, 0, s>>>(h_begin, n_hc, stride, state);
}
void launch_forces(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, Control* ctls, int respect_done, int n_sms,
                   int schedule, unsigned* queue) {
    // Schedule 0, persistent: one wave of FORCES_MINB blocks per SM taking
    // chunks from the queue (no tail). Schedule 1: a block per chunk, so
    // blocks retire all along and work on other streams (the next step's
    // contact pass) gets SMs while the kernel runs. Schedule 2 (3): the
    // persistent wave on all but 8 (16) SMs, which stay free for the side
    // streams' search. Without a queue, the persistent waves stride instead.
    const int free_sms = schedule == 2 ? 8 : schedule == 3 ? 16 : 0;
    long long cap = (long long)(n_sms > 2 * free_sms ? n_sms - free_sms : n_sms) * FORCES_MINB;
    if (schedule == 1) cap = GRID_CAP * 4;
    unsigned* q = schedule == 1 ? nullptr : queue;
    if (el.n_hc > 0)
        k_forces<<<active_grid(el.n_hc, 1, FORCES_TPB, cap), FORCES_TPB, 0, s>>>(el, nd, ctls, respect_done, q);
    if (el.n_sc > 0)
        k_forces_scalar<<<active_grid(el.n_sc, 1, SC_TPB, GRID_CAP), SC_TPB, 0, s>>>(el, nd, ctls, respect_done);
}
int forces_launches(const ElementArrays& el) { return (el.n_hc > 0 ? 1 : 0) + (el.n_sc > 0 ? 1 : 0); }
void launch_gather(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, double* f_out) {
    k_gather<<<(unsigned)blocks_for(nd.n, TPB), TPB, 0, s>>>(el, nd, f_out);
}
void launch_half(cudaStream_t s, const NodeArrays& nd, Control* ctls) {
    k_half<<<active_grid(nd.n, 3, TPB, GRID_CAP), TPB, 0, s>>>(nd, ctls);
}
void launch_full(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, Control* ctls) {
    k_full<<<active_grid(nd.n, 3, TPB, GRID_CAP), TPB, 0, s>>>(el, nd, ctls);
}
void launch_elem_dt(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, Control* ctls, const double* u, int respect_done,
                    long long e_begin) {
    if (el.n_all <= e_begin) return;
    k_elem_dt<<<active_grid(el.n_all - e_begin, 1, DT_TPB, GRID_CAP), DT_TPB, 0, s>>>(el, nd, ctls, u, respect_done, e_begin);
}
void launch_dt_finalize(cudaStream_t s, Control* ctls, int n_slots, int* mass_flag) {
    k_dt_finalize<<<(unsigned)blocks_for(n_slots, 128), 128, 0, s>>>(ctls, n_slots, mass_flag);
}
void launch_mass_scaling(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, Control* ctls, int force_apply) {
    k_mass_scaling<<<active_grid(nd.n, 1, TPB, GRID_CAP), TPB, 0, s>>>(el, nd, ctls, force_apply);
}
void launch_nonfinite(cudaStream_t s, const NodeArrays& nd, Control* ctls) {
    k_nonfinite<<<active_grid(nd.n, 1, TPB, GRID_CAP), TPB, 0, s>>>(nd, ctls);
}
void launch_build_active(cudaStream_t s, const ActiveBuild& b, const Control* ctls) {
    if (b.n_chunks <= 0) return;
    cudaMemsetAsync(b.counts, 0, sizeof(int) * ACTIVE_SPACES, s);
    k_build_active<<<(unsigned)blocks_for(b.n_chunks, TPB), TPB, 0, s>>>(b, ctls);
}
void launch_step_end(cudaStream_t s, Control* ctls, const ContactArrays& ca, const VehicleArrays& va, int check_separation,
                     int* done_out, int* mass_flag) {
    k_step_end<<<(unsigned)blocks_for(ca.n_slots, 128), 128, 0, s>>>(ctls, ca, va, check_separation, done_out, mass_flag);
}
void launch_fused(cudaStream_t s, const ElementArrays& el, const NodeArrays& nd, Control* ctls, const ContactArrays& ca,
                  const VehicleArrays& va, int* done_out, int* mass_flag, unsigned* block_counter) {
    k_fused<<<active_grid(nd.n, 3, TPB, GRID_CAP), TPB, 0, s>>>(el, nd, ctls, ca, va, done_out, mass_flag, block_counter);
}
void launch_vehicle_sums(cudaStream_t s, const VehicleArrays& va, const double* mass, const double* v, const double* v0, double* out) {
    if (va.n_vehicles <= 0) return;
    k_vehicle_sums<<<va.n_vehicles, VEH_TPB, 0, s>>>(va, mass, v, v0, out);
}
void launch_gather_ux(cudaStream_t s, long long n, const uint32_t* nodes, const double* u, double* out) {
    if (n <= 0) return;
    k_gather_ux<<<(unsigned)blocks_for(n, TPB), TPB, 0, s>>>(n, nodes, u, out);
}
void launch_vehicle_vx(cudaStream_t s, const VehicleArrays& va, const double* mass, const double* v, Control* ctls) {
    if (va.n_vehicles <= 0) return;
    k_vehicle_vx<<<(unsigned)(va.n_vehicles * va.vx_blocks), VEH_TPB, 0, s>>>(va, mass, v, ctls);
}

// Blocks per exhaustively searched contact: enough for about four blocks per
// SM over all such contacts (each block stages the contact's faces), at most 8.
unsigned brute_split(long long n_brute) {
    const long long target = 4 * 148;
    return (unsigned)std::min<long long>(8, std::max<long long>(1, (target + n_brute - 1) / std::max<long long>(n_brute, 1)));
}
// Few such contacts (a serving-size context): 16 lanes per primary node,
// each scanning every 16th face, and up to 16 blocks per contact, so that a
// node's scan is a quarter as long; many (a large batch): 4 lanes. Every
// choice finds the same first hit.
template <int LANES>
void launch_brute(cudaStream_t s, const ContactArrays& ca, const NodeArrays& nd, Control* ctls, const int* list, int single, unsigned n,
                  unsigned split, size_t smem) {
    k_contact_brute<LANES><<<dim3(n, split), BRUTE_TPB, smem, s>>>(ca, nd, ctls, list, single, list ? 1 : 0, 0.0, nullptr);
}
void launch_brute_any(cudaStream_t s, const ContactArrays& ca, const NodeArrays& nd, Control* ctls, const int* list, int single,
                      long long n_brute, size_t smem) {
    if (n_brute * 8 <= 4 * 148) {
        const unsigned split = (unsigned)std::min<long long>(16, std::max<long long>(1, (16 * 148 + n_brute - 1) / std::max<long long>(n_brute, 1)));
        launch_brute<16>(s, ca, nd, ctls, list, single, (unsigned)std::max<long long>(n_brute, 1), split, smem);
    } else {
        launch_brute<4>(s, ca, nd, ctls, list, single, (unsigned)n_brute, brute_split(n_brute), smem);
    }
}

void launch_contact_search(cudaStream_t s, const ContactArrays& ca, const NodeArrays& nd, Control* ctls, int c0, int c1, long long f0,
                           long long n_faces, long long n_slaves, long long bk0, long long bk1, int run_mode, int lanes,
                           cudaStream_t s_static) {
    (void)f0;
    if (c1 <= c0) return;
    // run: only moving faces (static ones keep their geometry); drop-in: every face of the range
    const uint32_t* list = run_mode ? ca.dyn_faces : nullptr;
    const long long n_list = run_mode ? ca.n_dyn_faces : n_faces;
    const Active act = run_mode ? ca.act_dynf : Active{nullptr, nullptr};
    const int do_grid = bk1 > bk0 && !ca.exhaustive ? 1 : 0;
    // Every search starts from clear grid bookkeeping (levels in use, entry
    // cursors, big-face list), whatever ran before it.
    cudaMemsetAsync(ca.grid_state, 0, sizeof(int) * (2 * (size_t)ca.contact_room + 1), s);
    if (n_list > 0)
        k_contact_faces<<<active_grid(n_list, FACE_LANES, FACE_TPB, GRID_CAP), FACE_TPB, 0, s>>>(ca, nd, ctls, c0, list, n_list,
                                                                                               run_mode, do_grid, act);
    if (do_grid) {
        k_grid_alloc<<<(unsigned)blocks_for(bk1 - bk0, TPB), TPB, 0, s>>>(ca, c0, c1);
        if (n_list > 0) {
            k_contact_insert<<<active_grid(n_list, 32, TPB, GRID_CAP), TPB, 0, s>>>(ca, c0, list, n_list, act);
            k_contact_big<<<(unsigned)(n_list < BIG_BLOCKS ? n_list : BIG_BLOCKS), BIG_TPB, 0, s>>>(ca, nd);
        }
    }
    // Exhaustive contacts: a block each (run: the listed ones; drop-in: the one contact if it is one).
    if (!ca.exhaustive) {
        if (run_mode && ca.n_brute > 0)
            launch_brute_any(s, ca, nd, ctls, ca.brute_contacts, 0, ca.n_brute, sizeof(FaceGeo) * ca.brute_max_faces);
        if (!run_mode && c1 == c0 + 1 && ca.is_brute_h && ca.is_brute_h[c0]) {
            launch_brute_any(s, ca, nd, ctls, nullptr, c0, 1, sizeof(FaceGeo) * BRUTE_MAX_FACES);
            n_slaves = 0;
        }
        if (run_mode) n_slaves = ca.n_grid_slaves;
    }
    // run: the listed entries (the static-grid ones apart); drop-in and
    // exhaustive: every entry of [c0, c1)
    const bool listed = run_mode && !ca.exhaustive;
    const uint32_t* slist = listed ? ca.grid_slaves : nullptr;
    const Active sact = listed ? ca.act_slave : Active{nullptr, nullptr};
    if (listed && ca.n_st_slaves > 0)
        k_contact_slaves<ST_LANES><<<active_grid(ca.n_st_slaves, ST_LANES, TPB, GRID_CAP), TPB, 0, s_static ? s_static : s>>>(
            ca, nd, ctls, c0, c1, run_mode, 0.0, nullptr, ca.n_st_slaves, ca.st_slaves, ca.act_stslave);
    if (n_slaves > 0) {
        const unsigned g = active_grid(n_slaves, lanes, TPB, GRID_CAP);
        switch (lanes) {
            case 1: k_contact_slaves<1><<<g, TPB, 0, s>>>(ca, nd, ctls, c0, c1, run_mode, 0.0, nullptr, n_slaves, slist, sact); break;
            case 2: k_contact_slaves<2><<<g, TPB, 0, s>>>(ca, nd, ctls, c0, c1, run_mode, 0.0, nullptr, n_slaves, slist, sact); break;
            case 4: k_contact_slaves<4><<<g, TPB, 0, s>>>(ca, nd, ctls, c0, c1, run_mode, 0.0, nullptr, n_slaves, slist, sact); break;
            case 8: k_contact_slaves<8><<<g, TPB, 0, s>>>(ca, nd, ctls, c0, c1, run_mode, 0.0, nullptr, n_slaves, slist, sact); break;
            case 16: k_contact_slaves<16><<<g, TPB, 0, s>>>(ca, nd, ctls, c0, c1, run_mode, 0.0, nullptr, n_slaves, slist, sact); break;
            default: k_contact_slaves<32><<<g, TPB, 0, s>>>(ca, nd, ctls, c0, c1, run_mode, 0.0, nullptr, n_slaves, slist, sact); break;
        }
    }
}

void launch_contact_finish(cudaStream_t s, const ContactArrays& ca, const NodeArrays& nd, Control* ctls, int c0, int c1, long long f0,
                           long long n_faces, long long n_slaves, double dt_override, const double* masses, double* f_out,
                           int skip_fixed, cudaStream_t s_heavy, cudaEvent_t ev_a, cudaEvent_t ev_b, cudaEvent_t ev_c, int next_step) {
    if (c1 <= c0) return;
    const int run_mode = dt_override > 0.0 ? 0 : 1;
    (void)f0;
    (void)n_faces;
    if (n_slaves > 0)
        k_contact_force<<<active_grid(n_slaves, FORCE_LANES, TPB, GRID_CAP), TPB, 0, s>>>(ca, ctls, c0, run_mode, dt_override, masses,
                                                                                         n_slaves, skip_fixed, next_step);
    long long nodes = ca.n_cnodes > 0 ? ca.n_cnodes : 1;
    // The heavy nodes (listed by the force pass) and the rest are disjoint:
    // with a second stream the two gathers run side by side.
    cudaStream_t sh = s_heavy ? s_heavy : s;
    if (s_heavy) {
        cudaEventRecord(ev_a, s);
        cudaStreamWaitEvent(sh, ev_a, 0);
    }
    k_contact_gather_heavy<<<(unsigned)(nodes < HEAVY_BLOCKS ? nodes : HEAVY_BLOCKS), HEAVY_TPB, 0, sh>>>(ca, nd, ctls, c0, c1, run_mode,
                                                                                                       f_out);
    if (s_heavy) cudaEventRecord(ev_b, sh);
    k_contact_gather<<<active_grid(nodes, 1, GATHER_TPB, GRID_CAP * 2), GATHER_TPB, 0, s>>>(ca, nd, ctls, c0, c1, run_mode, f_out,
                                                                                          skip_fixed);
    // The counts' reset follows both gathers: on the heavy stream it stays
    // off the caller's path (the caller joins that stream before its next
    // pass); the caller's stream waits only for the heavy sums.
    if (s_heavy) {
        cudaEventRecord(ev_c, s);
        cudaStreamWaitEvent(sh, ev_c, 0);
        k_contact_reset<<<1, RESET_TPB, 0, sh>>>(ca);
        cudaStreamWaitEvent(s, ev_b, 0);
    } else {
        k_contact_reset<<<1, RESET_TPB, 0, s>>>(ca);
    }
}

void launch_contact(cudaStream_t s, const ContactArrays& ca, const NodeArrays& nd, Control* ctls, int c0, int c1, long long f0,
                    long long n_faces, long long n_slaves, long long bk0, long long bk1, double dt_override, const double* masses,
                    double* f_out, int skip_fixed, int lanes) {
    launch_contact_search(s, ca, nd, ctls, c0, c1, f0, n_faces, n_slaves, bk0, bk1, dt_override > 0.0 ? 0 : 1, lanes);
    launch_contact_finish(s, ca, nd, ctls, c0, c1, f0, n_faces, n_slaves, dt_override, masses, f_out, skip_fixed);
}

int contact_search_launches(const ContactArrays& ca, bool run_mode, long long n_faces, long long n_slaves, long long bk0, long long bk1,
                            int c0) {
    int k = 0;
    const bool faces = (run_mode ? ca.n_dyn_faces : n_faces) > 0;
    if (faces) ++k;
    if (bk1 > bk0 && !ca.exhaustive) k += faces ? 3 : 1;
    if (!ca.exhaustive) {
        if (run_mode) {
            k += ca.n_brute > 0 ? 1 : 0;
            k += ca.n_st_slaves > 0 ? 1 : 0;
            n_slaves = ca.n_grid_slaves;
        } else if (ca.is_brute_h && ca.is_brute_h[c0]) {
            ++k;
            n_slaves = 0;
        }
    }
    if (n_slaves > 0) ++k;
    return k;
}

int contact_finish_launches(long long n_slaves) { return 3 + (n_slaves > 0 ? 1 : 0); }

int contact_launches(const ContactArrays& ca, bool run_mode, long long n_faces, long long n_slaves, long long bk0, long long bk1,
                     int c0) {
    return contact_search_launches(ca, run_mode, n_faces, n_slaves, bk0, bk1, c0) + contact_finish_launches(n_slaves);
}

void launch_contact_geometry(cudaStream_t s, const ContactArrays& ca, const NodeArrays& nd, int c0, int c1, long long f0,
                             long long n_faces) {
    (void)f0;
    if (c1 <= c0 || n_faces <= 0) return;
    (void)c1;
    k_contact_faces<<<active_grid(n_faces, FACE_LANES, FACE_TPB, GRID_CAP), FACE_TPB, 0, s>>>(ca, nd, nullptr, c0, nullptr, n_faces,
                                                                                            0, 0, Active{nullptr, nullptr});
}

}  // namespace crush

// ---------------------------------------------------------------------------
// Allocation-free contact call (crush_contact_apply_static): the primary-node
// filter of ContactRuntime::new (src/contact.rs:48-70) and one
// ContactRuntime::apply (src/contact.rs:92-160) for a single contact, with
// every intermediate in a fixed-size StaticContactScratch record. The search
// is exhaustive (no grid, whose table size would depend on the mesh), with
// the same narrow test, first-hit rule and force formula as the run's contact
// kernels; reactions are applied by node occurrence in the reference's order.
// ---------------------------------------------------------------------------
namespace crush {
namespace {

constexpr int STATIC_TPB = 256;
constexpr int STATIC_ONE_BLOCK = 1024;
constexpr int STATIC_TILE = 256;

// Single block: validates node ids, resets the record's counters and forms
// the filter box: the faces' bounding box at the reference positions grown by
// max_distance.
__global__ void __launch_bounds__(STATIC_ONE_BLOCK) k_static_prepare(StaticContactScratch* sc, long long n_model,
                                                                      const double* __restrict__ pos, long long n_nodes,
                                                                      const uint32_t* __restrict__ nodes, long long n_faces,
                                                                      const uint32_t* __restrict__ faces, double md) {
    __shared__ double s_lo[3][STATIC_ONE_BLOCK / 32], s_hi[3][STATIC_ONE_BLOCK / 32];
    __shared__ int s_bad;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    double lo[3] = {CUDART_INF, CUDART_INF, CUDART_INF}, hi[3] = {-CUDART_INF, -CUDART_INF, -CUDART_INF};
    int bad = 0;
    for (long long k = threadIdx.x; k < 4 * n_faces; k += blockDim.x) {
        const uint32_t n = faces[k];
        if (n >= n_model) {
            bad = 1;
            continue;
        }
        for (int d = 0; d < 3; ++d) {
            const double p = pos[3 * (long long)n + d];
            lo[d] = fmin(lo[d], p);
            hi[d] = fmax(hi[d], p);
        }
    }
    for (long long k = threadIdx.x; k < n_nodes; k += blockDim.x)
        if (nodes[k] >= n_model) bad = 1;
    if (bad) atomicOr(&s_bad, 1);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int d = 0; d < 3; ++d)
        for (int off = 16; off > 0; off >>= 1) {
            lo[d] = fmin(lo[d], __shfl_down_sync(0xffffffffu, lo[d], off));
            hi[d] = fmax(hi[d], __shfl_down_sync(0xffffffffu, hi[d], off));
        }
    if (lane == 0)
        for (int d = 0; d < 3; ++d) {
            s_lo[d][w] = lo[d];
            s_hi[d][w] = hi[d];
        }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int d = 0; d < 3; ++d) {
            double a = s_lo[d][0], b = s_hi[d][0];
            for (int k = 1; k < (int)(blockDim.x / 32); ++k) {
                a = fmin(a, s_lo[d][k]);
                b = fmax(b, s_hi[d][k]);
            }
            sc->box_lo[d] = a + -md;
            sc->box_hi[d] = b + md;
        }
        sc->pen_count = 0;
        sc->pen_max_bits = 0;
        sc->n_hits = 0;
        sc->error = s_bad;
    }
}

// Face geometry at X + u, thread per face (the arithmetic of k_contact_faces).
__global__ void k_static_faces(StaticContactScratch* sc, const double* __restrict__ pos, const double* __restrict__ u,
                               long long n_faces, const uint32_t* __restrict__ faces, double md) {
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n_faces || sc->error) return;
    FaceGeo g;
    for (int k = 0; k < 4; ++k) {
        const long long n = faces[4 * f + k];
        for (int d = 0; d < 3; ++d) g.x[k][d] = pos[3 * n + d] + u[3 * n + d];
    }
    double e1[3], e2[3];
    for (int d = 0; d < 3; ++d) {
        e1[d] = g.x[1][d] - g.x[0][d];
        e2[d] = g.x[2][d] - g.x[0][d];
    }
    const double nx = e1[1] * e2[2] - e1[2] * e2[1];
    const double ny = e1[2] * e2[0] - e1[0] * e2[2];
    const double nz = e1[0] * e2[1] - e1[1] * e2[0];
    const double len = sqrt(nx * nx + ny * ny + nz * nz);
    g.n[0] = nx / len;
    g.n[1] = ny / len;
    g.n[2] = nz / len;
    for (int d = 0; d < 3; ++d) {
        g.c[d] = (((g.x[0][d] + g.x[1][d]) + g.x[2][d]) + g.x[3][d]) / 4.0;
        double lo = g.x[0][d], hi = g.x[0][d];
        for (int k = 1; k < 4; ++k) {
            lo = fmin(lo, g.x[k][d]);
            hi = fmax(hi, g.x[k][d]);
        }
        g.lo[d] = lo + -md;
        g.hi[d] = hi + md;
    }
    sc->geo[f] = g;
}

// Warp per primary-node entry: the filter, then the smallest face index that
// passes the narrow test (the face the reference's in-order scan finds) and
// the penalty force on it.
__global__ void k_static_search(StaticContactScratch* sc, const double* __restrict__ pos, const double* __restrict__ u,
                                const double* __restrict__ masses, long long n_nodes, const uint32_t* __restrict__ nodes,
                                const double* __restrict__ node_scale, long long n_faces, double stiffness, double md,
                                double dt) {
    const long long s = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;  // warp-uniform
    const int lane = threadIdx.x & 31;
    if (s >= n_nodes || sc->error) return;
    const long long n = nodes[s];
    bool keep = true;
    for (int d = 0; d < 3; ++d) {
        const double x = pos[3 * n + d];
        if (!(x >= sc->box_lo[d] && x <= sc->box_hi[d])) keep = false;
    }
    if (!keep) {
        if (lane == 0) sc->hit[s] = -1;
        return;
    }
    const double p[3] = {pos[3 * n] + u[3 * n], pos[3 * n + 1] + u[3 * n + 1], pos[3 * n + 2] + u[3 * n + 2]};
    int best = INT_MAX;
    double best_sd = 0.0, sd;
    for (long long f = lane; f < n_faces; f += 32)
        if (f < best && face_hit(sc->geo[f], p, md, &sd)) {
            best = (int)f;
            best_sd = sd;
        }
    for (int off = 16; off > 0; off >>= 1) {
        const int ob = __shfl_down_sync(0xffffffffu, best, off);
        const double osd = __shfl_down_sync(0xffffffffu, best_sd, off);
        if (ob < best) {
            best = ob;
            best_sd = osd;
        }
    }
    if (lane != 0) return;
    if (best == INT_MAX) {
        sc->hit[s] = -1;
        return;
    }
    const double scale = node_scale ? node_scale[s] : 1.0;
    const double m = masses[n];
    const double depth = fmin(-best_sd, 0.1 * md);
    const double k_pen = fmin(stiffness * scale, 0.1 * m / (dt * dt));
    const double mag = fmin(k_pen * depth, m * 1.0e5);
    const FaceGeo& g = sc->geo[best];
    sc->hit[s] = best;
    sc->hit_force[3 * s] = mag * g.n[0];
    sc->hit_force[3 * s + 1] = mag * g.n[1];
    sc->hit_force[3 * s + 2] = mag * g.n[2];
    atomicAdd(&sc->pen_count, 1ull);
    atomicMax(&sc->pen_max_bits, (unsigned long long)__double_as_longlong(-best_sd + 0.0));  // + 0.0: no -0.0 bits
}

// Single block: the entries that hit, compacted in entry order.
__global__ void __launch_bounds__(STATIC_ONE_BLOCK) k_static_compact(StaticContactScratch* sc, long long n_nodes) {
    __shared__ int s_warp[STATIC_ONE_BLOCK / 32];
    __shared__ int s_base;
    if (sc->error) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) s_base = 0;
    __syncthreads();
    for (long long c0 = 0; c0 < n_nodes; c0 += blockDim.x) {
        const long long i = c0 + threadIdx.x;
        const bool flag = i < n_nodes && sc->hit[i] >= 0;
        const unsigned ballot = __ballot_sync(0xffffffffu, flag);
        if (lane == 0) s_warp[w] = __popc(ballot);
        __syncthreads();
        int before = 0, total = 0;
        for (int k = 0; k < nw; ++k) {
            if (k < w) before += s_warp[k];
            total += s_warp[k];
        }
        if (flag) sc->hit_list[s_base + before + __popc(ballot & ((1u << lane) - 1u))] = (int)i;
        __syncthreads();
        if (threadIdx.x == 0) s_base += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) sc->n_hits = s_base;
}

// Thread per node occurrence (the primary-node entries, then the face
// corners): the node's force value after this contact, adding the hits in
// entry order — +F for its own hit, -F/4 per corner it fills on a hit face —
// starting from the value in f_accum (src/contact.rs:146-153).
__global__ void __launch_bounds__(STATIC_TPB) k_static_occ(StaticContactScratch* sc, long long n_nodes, const uint32_t* __restrict__ nodes,
                                                           long long n_faces, const uint32_t* __restrict__ faces,
                                                           const double* __restrict__ f_accum) {
    __shared__ uint32_t t_node[STATIC_TILE];
    __shared__ uint32_t t_face[STATIC_TILE][4];
    __shared__ double t_f[STATIC_TILE][3];
    if (sc->error) return;  // grid-uniform
    const long long n_occ = n_nodes + 4 * n_faces;
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = o < n_occ;
    const long long n = live ? (long long)(o < n_nodes ? nodes[o] : faces[o - n_nodes]) : 0;
    double v0 = 0.0, v1 = 0.0, v2 = 0.0;
    if (live) {
        v0 = f_accum[3 * n];
        v1 = f_accum[3 * n + 1];
        v2 = f_accum[3 * n + 2];
    }
    const int H = sc->n_hits;
    for (int t0 = 0; t0 < H; t0 += STATIC_TILE) {
        const int nt = min(STATIC_TILE, H - t0);
        __syncthreads();
        for (int k = threadIdx.x; k < nt; k += blockDim.x) {
            const int s = sc->hit_list[t0 + k];
            const long long fc = sc->hit[s];
            t_node[k] = nodes[s];
            for (int j = 0; j < 4; ++j) t_face[k][j] = faces[4 * fc + j];
            for (int d = 0; d < 3; ++d) t_f[k][d] = sc->hit_force[3 * s + d];
        }
        __syncthreads();
        if (live)
            for (int k = 0; k < nt; ++k) {
                if (t_node[k] == (uint32_t)n) {
                    v0 += t_f[k][0];
                    v1 += t_f[k][1];
                    v2 += t_f[k][2];
                }
                for (int j = 0; j < 4; ++j)
                    if (t_face[k][j] == (uint32_t)n) {
                        v0 -= 0.25 * t_f[k][0];
                        v1 -= 0.25 * t_f[k][1];
                        v2 -= 0.25 * t_f[k][2];
                    }
            }
    }
    if (live) {
        sc->occ[3 * o] = v0;
        sc->occ[3 * o + 1] = v1;
        sc->occ[3 * o + 2] = v2;
    }
}

// Thread per occurrence: store the node's new value (every occurrence of a
// node holds the same value, so repeated stores agree); thread 0 reports.
__global__ void k_static_write(StaticContactScratch* sc, long long n_nodes, const uint32_t* __restrict__ nodes, long long n_faces,
                               const uint32_t* __restrict__ faces, double* __restrict__ f_accum, int64_t* stats_count,
                               double* stats_max, int* stats_status) {
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int err = sc->error;
    if (o == 0) {
        if (stats_count) *stats_count = err ? 0 : (int64_t)sc->pen_count;
        if (stats_max) *stats_max = err ? 0.0 : __longlong_as_double((long long)sc->pen_max_bits);
        if (stats_status) *stats_status = err ? -1 : 0;  // CRUSH_ERR_INVALID / CRUSH_OK
    }
    if (err || o >= n_nodes + 4 * n_faces) return;
    const long long n = o < n_nodes ? nodes[o] : faces[o - n_nodes];
    f_accum[3 * n] = sc->occ[3 * o];
    f_accum[3 * n + 1] = sc->occ[3 * o + 1];
    f_accum[3 * n + 2] = sc->occ[3 * o + 2];
}

}  // namespace

void launch_contact_static(cudaStream_t s, StaticContactScratch* sc, long long n_model_nodes, const double* pos, const double* u,
                           const double* masses, long long n_nodes, const uint32_t* nodes, const double* node_scale,
                           long long n_faces, const uint32_t* faces, double stiffness, double max_distance, double dt,
                           double* f_accum, int64_t* stats_count, double* stats_max, int* stats_status) {
    k_static_prepare<<<1, STATIC_ONE_BLOCK, 0, s>>>(sc, n_model_nodes, pos, n_nodes, nodes, n_faces, faces, max_distance);
    if (n_faces > 0) k_static_faces<<<(unsigned)blocks_for(n_faces, STATIC_TPB), STATIC_TPB, 0, s>>>(sc, pos, u, n_faces, faces, max_distance);
    if (n_nodes > 0)
        k_static_search<<<(unsigned)blocks_for(n_nodes * 32, STATIC_TPB), STATIC_TPB, 0, s>>>(
            sc, pos, u, masses, n_nodes, nodes, node_scale, n_faces, stiffness, max_distance, dt);
    k_static_compact<<<1, STATIC_ONE_BLOCK, 0, s>>>(sc, n_nodes);
    const long long n_occ = n_nodes + 4 * n_faces;
    if (n_occ > 0) k_static_occ<<<(unsigned)blocks_for(n_occ, STATIC_TPB), STATIC_TPB, 0, s>>>(sc, n_nodes, nodes, n_faces, faces, f_accum);
    k_static_write<<<(unsigned)blocks_for(n_occ > 0 ? n_occ : 1, STATIC_TPB), STATIC_TPB, 0, s>>>(
        sc, n_nodes, nodes, n_faces, faces, f_accum, stats_count, stats_max, stats_status);
}

}  // namespace crush
