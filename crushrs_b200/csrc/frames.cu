// frames.cu — frames on the device: every frame_steps steps the nodal
// displacement and, per element, plastic strain, Cauchy stress and erosion
// (Frame and its capture in crushrs::run, src/solver.rs:52-60, :265-281,
// :345-348, :353-355; plastic_strain and cauchy_stress, src/kernel.rs:269-321),
// copied into device buffers sized at configuration.
#include "kernels.cuh"
#include "hencky.cuh"

namespace crush {

namespace {

constexpr int FRAME_TPB = 256;

// Whether slot `slot` takes a frame now (the history rule: the run's first
// frame, a multiple of frame_steps, or the last step of a finished crash).
__device__ __forceinline__ bool frame_due(const FrameArrays& f, const Control* ctl, int slot, int mode) {
    if (!f.slot_on[slot]) return false;
    if (mode == HIST_INITIAL) return true;
    if (ctl->step == f.last_step[slot]) return false;
    return mode == HIST_FINAL ? ctl->done != 0 : ctl->step % f.steps == 0;
}

// blockIdx.y = slot: its 3 n displacement values as f32.
__global__ void __launch_bounds__(FRAME_TPB) k_frame_nodes(FrameArrays f, const double* __restrict__ u, const Control* ctls, int mode) {
    const int slot = blockIdx.y;
    if (!frame_due(f, ctls + slot, slot, mode)) return;
    const long long r = f.count[slot];
    if (r >= f.slot_max[slot]) return;
    const long long n3 = 3 * f.n_nodes[slot], u0 = 3 * f.node0[slot];
    float* out = f.disp + f.disp_base[slot] + r * n3;
    for (long long i = (long long)blockIdx.x * FRAME_TPB + threadIdx.x; i < n3; i += (long long)gridDim.x * FRAME_TPB)
        out[i] = (float)u[u0 + i];
}

// blockIdx.y = slot: per element the erosion flag, the plastic strain
// (compaction of a honeycomb element, 0 for an elastic one) and the Cauchy
// stress: R sigma_hat R^T from the committed f32 state in f64 for a
// honeycomb element, as src/kernel.rs:285-293 computes it; tau / J of the
// Hencky stress at the current F for an elastic one (:294-315); 0 when
// eroded or inverted.
__global__ void __launch_bounds__(FRAME_TPB) k_frame_elems(FrameArrays f, const double* __restrict__ u, const Control* ctls, int mode) {
    const int slot = blockIdx.y;
    if (!frame_due(f, ctls + slot, slot, mode)) return;
    const long long r = f.count[slot];
    if (r >= f.slot_max[slot]) return;
    const long long ne = f.n_elems[slot], e0 = f.elem0[slot];
    const long long base = f.elem_base[slot] + r * ne;
    for (long long i = (long long)blockIdx.x * FRAME_TPB + threadIdx.x; i < ne; i += (long long)gridDim.x * FRAME_TPB) {
        const long long e = e0 + i;
        const bool er = f.eroded_all[e] != 0;
        const long long h = f.hc_index[e];
        float ps = 0.0f, c6[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (h >= 0) {
            float st[28];
            for (int q = 0; q < 7; ++q) {
                const float4 v = f.state[q * f.state_stride + h];
                st[4 * q] = v.x;
                st[4 * q + 1] = v.y;
                st[4 * q + 2] = v.z;
                st[4 * q + 3] = v.w;
            }
            ps = st[S_COMPACTION];
            if (!er) {
                double R[3][3], sh[3][3], a[3][3];
                for (int i2 = 0; i2 < 3; ++i2)
                    for (int j = 0; j < 3; ++j) R[i2][j] = (double)st[9 + 3 * i2 + j];
                const double s0 = st[18], s1 = st[19], s2 = st[20], s3 = st[21], s4 = st[22], s5 = st[23];
                sh[0][0] = s0; sh[0][1] = s3; sh[0][2] = s5;
                sh[1][0] = s3; sh[1][1] = s1; sh[1][2] = s4;
                sh[2][0] = s5; sh[2][1] = s4; sh[2][2] = s2;
                for (int i2 = 0; i2 < 3; ++i2)
                    for (int j = 0; j < 3; ++j) a[i2][j] = R[i2][0] * sh[0][j] + R[i2][1] * sh[1][j] + R[i2][2] * sh[2][j];
                double c[3][3];
                for (int i2 = 0; i2 < 3; ++i2)
                    for (int j = 0; j < 3; ++j) c[i2][j] = a[i2][0] * R[j][0] + a[i2][1] * R[j][1] + a[i2][2] * R[j][2];
                c6[0] = (float)c[0][0];
                c6[1] = (float)c[1][1];
                c6[2] = (float)c[2][2];
                c6[3] = (float)c[0][1];
                c6[4] = (float)c[1][2];
                c6[5] = (float)c[0][2];
            }
        } else if (f.sc_index && !er) {
            const long long q = f.sc_index[e];
            double fm[9];
            for (int k = 0; k < 9; ++k) fm[k] = 0.0;
            for (int k = 0; k < 8; ++k) {
                const long long n = f.conn_all[8 * e + k];
                for (int a = 0; a < 3; ++a) {
                    const double xa = f.pos[3 * n + a] + u[3 * n + a];
                    for (int b = 0; b < 3; ++b) fm[3 * a + b] += xa * f.sc_geo[(SC_GRAD + 3 * k + b) * f.n_sc + q];
                }
            }
            const double j = fm[0] * (fm[4] * fm[8] - fm[7] * fm[5]) - fm[1] * (fm[3] * fm[8] - fm[6] * fm[5]) +
                             fm[2] * (fm[3] * fm[7] - fm[6] * fm[4]);
            if (j > 0.0) {
                double tau[9];
                hencky_elastic(f.sc_mat[2 * q], f.sc_mat[2 * q + 1], fm, tau);
                c6[0] = (float)(tau[0] / j);
                c6[1] = (float)(tau[4] / j);
                c6[2] = (float)(tau[8] / j);
                c6[3] = (float)(tau[1] / j);
                c6[4] = (float)(tau[5] / j);
                c6[5] = (float)(tau[2] / j);
            }
        }
        f.eroded[base + i] = er ? 1 : 0;
        f.pstrain[base + i] = ps;
        for (int k = 0; k < 6; ++k) f.stress[6 * (base + i) + k] = c6[k];
    }
}

__global__ void k_frame_finish(FrameArrays f, const Control* ctls, int mode) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= f.n_slots) return;
    const Control* ctl = ctls + slot;
    if (!frame_due(f, ctl, slot, mode)) return;
    const long long r = f.count[slot];
    if (r < f.slot_max[slot]) {
        f.time[slot * f.stride + r] = ctl->t;
        f.step[slot * f.stride + r] = ctl->step;
    }
    f.count[slot] = r + 1;
    f.last_step[slot] = ctl->step;
}

}  // namespace

void launch_frames(cudaStream_t s, const FrameArrays& f, const double* u, const Control* ctls, int mode) {
    k_frame_nodes<<<dim3((unsigned)f.node_blocks, (unsigned)f.n_slots), FRAME_TPB, 0, s>>>(f, u, ctls, mode);
    k_frame_elems<<<dim3((unsigned)f.elem_blocks, (unsigned)f.n_slots), FRAME_TPB, 0, s>>>(f, u, ctls, mode);
    k_frame_finish<<<(unsigned)((f.n_slots + 127) / 128), 128, 0, s>>>(f, ctls, mode);
}

}  // namespace crush
