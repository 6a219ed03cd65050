// history.cu — time histories on the device: per-part states and
// accelerometer node samples, recorded inside the step sequence every
// history_steps steps (src/solver.rs:114-187 part_states and
// sample_accelerometers, called at :283-286 and :349-358), so a run that
// records every step needs no device-to-host copy per step.
#include "kernels.cuh"

namespace crush {

namespace {

constexpr int HIST_TPB = 256;

// Whether slot `slot` takes a record now: its run's first record, a step
// that is a multiple of history_steps, or the last step of a finished crash;
// never twice at one step.
__device__ __forceinline__ bool hist_due(const HistoryArrays& h, const Control* ctl, int slot, int mode) {
    if (!h.slot_on[slot]) return false;
    if (mode == HIST_INITIAL) return true;
    if (ctl->step == h.last_step[slot]) return false;
    return mode == HIST_FINAL ? ctl->done != 0 : ctl->step % h.steps == 0;
}

// Nodal acceleration (net force / mass, with the added mass of mass
// scaling), zero at fixed nodes (src/solver.rs:333-341).
__device__ __forceinline__ double hist_acc(const NodeArrays& nd, const double* __restrict__ f_ext, long long n, int d) {
    if (nd.fixed[n]) return 0.0;
    const long long k = 3 * n + d;
    return (f_ext[k] - nd.f_int[k]) * nd.inv_mass[n];
}

__device__ __forceinline__ void cross3(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ __forceinline__ double norm3(const double* a) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

// Body-fixed axes from three nodes at X + u (LocalFrame::axes,
// src/model.rs:45-61): e1 along origin -> x_axis, e3 normal to the plane of
// e1 and origin -> plane, e2 = e3 x e1; degenerate inputs fall back to the
// global axes as there. Rows are the axes.
__device__ void frame_axes(const NodeArrays& nd, const uint32_t* fn, double ax[3][3]) {
    double o[3], e1[3], p[3];
    for (int d = 0; d < 3; ++d) {
        o[d] = nd.pos[3ll * fn[0] + d] + nd.u[3ll * fn[0] + d];
        e1[d] = (nd.pos[3ll * fn[1] + d] + nd.u[3ll * fn[1] + d]) - o[d];
        p[d] = (nd.pos[3ll * fn[2] + d] + nd.u[3ll * fn[2] + d]) - o[d];
    }
    if (norm3(e1) < 1e-300) {
        e1[0] = 1.0;
        e1[1] = 0.0;
        e1[2] = 0.0;
    }
    const double n1 = norm3(e1);
    for (int d = 0; d < 3; ++d) e1[d] /= n1;
    double c[3];
    cross3(p, e1, c);
    if (norm3(c) < 1e-12 * fmax(norm3(p), 1e-300)) {
        const bool use_x = fabs(e1[0]) < 0.9;
        p[0] = use_x ? 1.0 : 0.0;
        p[1] = use_x ? 0.0 : 1.0;
        p[2] = 0.0;
    }
    double e3[3], e2[3];
    cross3(e1, p, e3);
    const double n3 = norm3(e3);
    for (int d = 0; d < 3; ++d) e3[d] /= n3;
    cross3(e3, e1, e2);
    for (int d = 0; d < 3; ++d) {
        ax[0][d] = e1[d];
        ax[1][d] = e2[d];
        ax[2][d] = e3[d];
    }
}

// Block (part unit, chunk b): mass-weighted sums over the chunk's nodes,
// reduced in a fixed order into partial[pu][b].
__global__ void __launch_bounds__(HIST_TPB) k_hist_parts(HistoryArrays h, NodeArrays nd, const Control* ctls,
                                                         const double* __restrict__ f_ext, int mode, const double* __restrict__ f_ext_odd) {
    __shared__ double sh[HIST_PART_VALUES][HIST_TPB];
    const int pu = blockIdx.x / HIST_BLOCKS, b = blockIdx.x % HIST_BLOCKS;
    const int slot = h.pu_slot[pu];
    if (!hist_due(h, ctls + slot, slot, mode)) return;  // block-uniform
    if (mode == HIST_FINAL && f_ext_odd && ((ctls[slot].step - 1) & 1)) f_ext = f_ext_odd;
    const long long lo = h.pu_off[pu], len = (long long)h.pu_off[pu + 1] - lo;
    const long long per = (len + HIST_BLOCKS - 1) / HIST_BLOCKS;
    const long long i0 = lo + b * per, i1 = min(lo + len, i0 + per);
    double acc[HIST_PART_VALUES];
#pragma unroll
    for (int k = 0; k < HIST_PART_VALUES; ++k) acc[k] = 0.0;
    for (long long i = i0 + threadIdx.x; i < i1; i += HIST_TPB) {
        const long long n = h.pu_nodes[i];
        const double m = nd.mass[n];
        acc[0] += m;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double v = nd.v[3 * n + d];
            acc[1 + d] += m * v;
            acc[4 + d] += m * nd.u[3 * n + d];
            acc[7 + d] += m * hist_acc(nd, f_ext, n, d);
            acc[10] += 0.5 * m * v * v;
        }
    }
#pragma unroll
    for (int k = 0; k < HIST_PART_VALUES; ++k) sh[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int off = HIST_TPB / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off)
#pragma unroll
            for (int k = 0; k < HIST_PART_VALUES; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x < HIST_PART_VALUES) h.partial[((long long)pu * HIST_BLOCKS + b) * HIST_PART_VALUES + threadIdx.x] = sh[threadIdx.x][0];
}

// Block per slot: the record's part states (partials added in block order,
// then divided by the mass as src/solver.rs:131-139 does) and accelerometer
// samples, its time and step, and the slot's record count.
__global__ void __launch_bounds__(HIST_TPB) k_hist_finish(HistoryArrays h, NodeArrays nd, const Control* ctls,
                                                          const double* __restrict__ f_ext, int mode, const double* __restrict__ f_ext_odd) {
    const int slot = blockIdx.x;
    const Control* ctl = ctls + slot;
    if (!hist_due(h, ctl, slot, mode)) return;  // block-uniform
    if (mode == HIST_FINAL && f_ext_odd && ((ctl->step - 1) & 1)) f_ext = f_ext_odd;
    const long long r = h.rec_count[slot];
    const bool keep = r < h.slot_max[slot];
    if (keep) {
        for (int pu = h.slot_pu_off[slot] + threadIdx.x; pu < h.slot_pu_off[slot + 1]; pu += HIST_TPB) {
            double s[HIST_PART_VALUES];
            for (int k = 0; k < HIST_PART_VALUES; ++k) s[k] = 0.0;
            for (int b = 0; b < HIST_BLOCKS; ++b)
                for (int k = 0; k < HIST_PART_VALUES; ++k) s[k] += h.partial[((long long)pu * HIST_BLOCKS + b) * HIST_PART_VALUES + k];
            const double inv = s[0] > 0.0 ? 1.0 / s[0] : 0.0;
            double* o = h.part_rec + ((long long)pu * h.max_rec + r) * HIST_PART_VALUES;
            o[0] = s[0];
            for (int k = 1; k < 10; ++k) o[k] = s[k] * inv;
            o[10] = s[10];
        }
        for (int j = h.slot_an_off[slot] + threadIdx.x; j < h.slot_an_off[slot + 1]; j += HIST_TPB) {
            const long long n = h.an_node[j];
            double x[3], u[3], v[3], a[3];
            for (int d = 0; d < 3; ++d) {
                u[d] = nd.u[3 * n + d];
                x[d] = nd.pos[3 * n + d] + u[d];
                v[d] = nd.v[3 * n + d];
                a[d] = hist_acc(nd, f_ext, n, d);
            }
            double* o = h.node_rec + ((long long)j * h.max_rec + r) * HIST_NODE_VALUES;
            for (int d = 0; d < 3; ++d) {
                o[d] = x[d];
                o[3 + d] = u[d];
                o[6 + d] = v[d];
                o[9 + d] = a[d];
            }
            const int f = h.an_frame[j];
            if (f < 0) {
                for (int d = 0; d < 3; ++d) {
                    o[12 + d] = u[d];
                    o[15 + d] = v[d];
                    o[18 + d] = a[d];
                }
            } else {
                double ax[3][3];
                frame_axes(nd, h.fr_nodes + 3ll * f, ax);
                for (int i = 0; i < 3; ++i) {  // rotate, src/solver.rs:143-145
                    o[12 + i] = ax[i][0] * u[0] + ax[i][1] * u[1] + ax[i][2] * u[2];
                    o[15 + i] = ax[i][0] * v[0] + ax[i][1] * v[1] + ax[i][2] * v[2];
                    o[18 + i] = ax[i][0] * a[0] + ax[i][1] * a[1] + ax[i][2] * a[2];
                }
            }
        }
    }
    __syncthreads();  // every thread has read rec_count
    if (threadIdx.x == 0) {
        if (keep) {
            h.rec_time[(long long)slot * h.max_rec + r] = ctl->t;
            h.rec_step[(long long)slot * h.max_rec + r] = ctl->step;
        }
        h.rec_count[slot] = r + 1;
        h.last_step[slot] = ctl->step;
    }
}

}  // namespace

void launch_history(cudaStream_t s, const HistoryArrays& h, const NodeArrays& nd, const Control* ctls, const double* f_ext, int mode,
                    const double* f_ext_odd) {
    if (h.n_pu > 0) k_hist_parts<<<(unsigned)(h.n_pu * HIST_BLOCKS), HIST_TPB, 0, s>>>(h, nd, ctls, f_ext, mode, f_ext_odd);
    k_hist_finish<<<(unsigned)h.n_slots, HIST_TPB, 0, s>>>(h, nd, ctls, f_ext, mode, f_ext_odd);
}

}  // namespace crush
