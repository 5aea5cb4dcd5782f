// integrate.cu — integrators, energy minimisation step and state transfer.
//
// Replaces the integration part of CompoundIntegrationKernel
// (code/LIMA_ENGINE/src/EngineKernels.cuh:344-441):
//   velocity Verlet as in EngineUtils::integrateVelocityVVS / integratePositionVVS
//   (code/LIMA_ENGINE/src/EngineUtils.cuh:31-41):
//       v = v_prev + (F + F_prev) dt/2m ; x += v dt + F dt^2/2m ; v_prev = v * scale
//   leapfrog (the native integrator): v += F dt/m ; x += v dt
// Positions are updated in FP64 relative to the box origin (the reference keeps
// int32 fixed point relative to per-compound integer origins,
// code/LIMA_BASE/include/LimaTypes.cuh:297-334); the float4 working copy used by
// the force kernels is refreshed from the FP64 value.
// The energy-minimisation step restates IntegratePositionADAM and
// ForceActivationFunction (EngineUtils.cuh:44-72,112-140).
#include "engine.h"

namespace lima {

__device__ __forceinline__ float3 load_force(const DevState& st, int s) {
    const double inv = 1.0 / FORCE_SCALE;
    return make_float3((float)((double)st.fx[s] * inv), (float)((double)st.fy[s] * inv),
                       (float)((double)st.fz[s] * inv));
}

// Flags a force accumulator at or beyond half the int64 range (2^30 J/mol/nm):
// a single contribution there has saturated its conversion and a sum may wrap,
// so the step's forces cannot be trusted (LIMA_STATUS_FORCE_SATURATED).
__device__ __forceinline__ void check_saturation(const DevState& st, int s) {
    constexpr long long LIM = 1ll << 62;
    const long long x = st.fx[s], y = st.fy[s], z = st.fz[s];
    if (x >= LIM || x <= -LIM || y >= LIM || y <= -LIM || z >= LIM || z <= -LIM)
        atomicOr(st.status, ST_FORCE_SATURATED);
}

// Every load of a slot is issued before the padding test (padding slots hold
// valid memory), so the per-slot loads form one round of memory latency
// instead of a chain behind the slot's `orig` entry.
template <int INTEGRATOR, bool ENERGY>
__global__ void k_integrate(DevState st, IntegrateParams p) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double ke = 0.0;
    int sysi = -1;
    if (s < st.n_slots) {
        const int o = st.orig[s];
        const int sy = st.cluster_sys[s / CLUSTER];
        const float3 F = load_force(st, s);
        float4 v = st.vel[s];
        const double px = st.px[s], py = st.py[s], pz = st.pz[s];
        const float q = st.xyzq[s].w;
        const float4 r = st.xyz_ref[s];
        const float4 fp = INTEGRATOR == 0 ? make_float4(0.f, 0.f, 0.f, 0.f) : st.fprev[s];
        const float scale = st.vscale[sy];
        if (o >= 0) {
            sysi = sy;
            const float im = v.w;
            const float dt = (float)p.dt;
            if (!(isfinite(F.x) && isfinite(F.y) && isfinite(F.z))) atomicOr(st.status, ST_NONFINITE);
            check_saturation(st, s);
            double dx, dy, dz;
            if (INTEGRATOR == 0) {
                const float m = im > 0.f ? 1.f / im : 0.f;
                const float vx = (v.x + F.x * im * dt) * scale;
                const float vy = (v.y + F.y * im * dt) * scale;
                const float vz = (v.z + F.z * im * dt) * scale;
                if (ENERGY) {
                    // average of the two half-step kinetic energies
                    ke = 0.25 * (double)m * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z +
                                             (double)vx * vx + (double)vy * vy + (double)vz * vz);
                }
                v.x = vx;
                v.y = vy;
                v.z = vz;
                dx = (double)vx * p.dt;
                dy = (double)vy * p.dt;
                dz = (double)vz * p.dt;
            } else {
                const float h = 0.5f * dt * im;
                const float vx = v.x + (F.x + fp.x) * h;
                const float vy = v.y + (F.y + fp.y) * h;
                const float vz = v.z + (F.z + fp.z) * h;
                if (ENERGY) {
                    const float m = im > 0.f ? 1.f / im : 0.f;
                    ke = 0.5 * (double)m * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
                }
                const float a = 0.5f * im * dt * dt;
                dx = (double)vx * p.dt + (double)(F.x * a);
                dy = (double)vy * p.dt + (double)(F.y * a);
                dz = (double)vz * p.dt + (double)(F.z * a);
                st.fprev[s] = make_float4(F.x, F.y, F.z, 0.f);
                v.x = vx * scale;
                v.y = vy * scale;
                v.z = vz * scale;
            }
            st.vel[s] = v;
            const double x = px + dx, y = py + dy, z = pz + dz;
            st.px[s] = x;
            st.py[s] = y;
            st.pz[s] = z;
            st.xyzq[s] = make_float4((float)x, (float)y, (float)z, q);
            // an atom beyond half the Verlet buffer from its position at the list
            // build may meet a partner the list does not hold
            const float ex = (float)x - r.x, ey = (float)y - r.y, ez = (float)z - r.z;
            if (ex * ex + ey * ey + ez * ez > p.half_skin2) atomicOr(st.status, ST_MOVED_TOO_FAR);
        }
    }
    if (ENERGY) add_energy_fixed(st.energy, sysi, ke, E_KINETIC);
}

int launch_integrate(const DevState& st, const IntegrateParams& p, bool energy, cudaStream_t s) {
    const int TB = 256;
    const int g = (st.n_slots + TB - 1) / TB;
    if (p.integrator == 0) {
        if (energy) k_integrate<0, true><<<g, TB, 0, s>>>(st, p);
        else k_integrate<0, false><<<g, TB, 0, s>>>(st, p);
    } else {
        if (energy) k_integrate<1, true><<<g, TB, 0, s>>>(st, p);
        else k_integrate<1, false><<<g, TB, 0, s>>>(st, p);
    }
    return 1;
}

// ADAM step on tanh-clamped forces; positions move by alpha*mhat/(sqrt(vhat)+eps)*1e-8 nm
__global__ void k_em_step(DevState st, int step) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= st.n_slots || st.orig[s] < 0) return;
    check_saturation(st, s);
    float3 F = load_force(st, s);
    const float fmax = 1.0e6f;  // 1000 kJ/mol/nm
    const float fl = sqrtf(F.x * F.x + F.y * F.y + F.z * F.z);
    const float sc = fmax * tanhf(fl / fmax) / (fl + 1e-8f);
    const float g[3] = {F.x * sc * 1e-8f, F.y * sc * 1e-8f, F.z * sc * 1e-8f};
    float4 m = st.adam_m[s], v = st.adam_v[s];
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f / (1.f - powf(b1, (float)step));
    const float c2 = 1.f / (1.f - powf(b2, (float)step));
    float* mm = &m.x;
    float* vv = &v.x;
    double d[3];
    for (int k = 0; k < 3; ++k) {
        mm[k] = mm[k] * b1 + g[k] * (1.f - b1);
        vv[k] = vv[k] * b2 + g[k] * g[k] * (1.f - b2);
        d[k] = (double)(mm[k] * c1 / (sqrtf(vv[k] * c2) + 1e-8f) * 8000.f) * 1e-8;
    }
    st.adam_m[s] = m;
    st.adam_v[s] = v;
    const double x = st.px[s] + d[0], y = st.py[s] + d[1], z = st.pz[s] + d[2];
    st.px[s] = x;
    st.py[s] = y;
    st.pz[s] = z;
    const float q = st.xyzq[s].w;
    st.xyzq[s] = make_float4((float)x, (float)y, (float)z, q);
}

int launch_em_step(const DevState& st, int step, float* /*max_force_out_dev*/, cudaStream_t s) {
    const int TB = 256;
    k_em_step<<<(st.n_slots + TB - 1) / TB, TB, 0, s>>>(st, step);
    return 1;
}

// per-atom maximum |F| (as float bits; non-negative floats order like ints)
__global__ void k_max_force(DevState st, float* out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    float fl = 0.f;
    if (s < st.n_slots && st.orig[s] >= 0) {
        const float3 F = load_force(st, s);
        fl = sqrtf(F.x * F.x + F.y * F.y + F.z * F.z);
        if (!isfinite(fl)) fl = 3.0e38f;
    }
    for (int o = 16; o > 0; o >>= 1) fl = fmaxf(fl, __shfl_xor_sync(0xffffffffu, fl, o));
    if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int*>(out), __float_as_int(fl));
}

int launch_max_force(const DevState& st, float* out, cudaStream_t s) {
    const int TB = 256;
    k_max_force<<<(st.n_slots + TB - 1) / TB, TB, 0, s>>>(st, out);
    return 1;
}

// slot order -> original order
__global__ void k_gather_state(DevState st, double* pos, float* vel) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= st.n_atoms) return;
    const int s = st.slot_of[a];
    if (pos) {
        pos[3 * a] = st.px[s];
        pos[3 * a + 1] = st.py[s];
        pos[3 * a + 2] = st.pz[s];
    }
    if (vel) {
        const float4 v = st.vel[s];
        vel[3 * a] = v.x;
        vel[3 * a + 1] = v.y;
        vel[3 * a + 2] = v.z;
    }
}

// kinetic energy per system from the stored velocities (thermostat measurement)
__global__ void k_kinetic(DevState st, long long* ke) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    int sysi = -1;
    if (s < st.n_slots && st.orig[s] >= 0) {
        sysi = st.cluster_sys[s / CLUSTER];
        const float4 v = st.vel[s];
        const double m = v.w > 0.f ? 1.0 / (double)v.w : 0.0;
        e = 0.5 * m * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
    }
    add_energy_fixed(ke, sysi, e, E_KINETIC);
}

int launch_kinetic(const DevState& st, long long* ke, cudaStream_t s) {
    const int TB = 256;
    k_kinetic<<<(st.n_slots + TB - 1) / TB, TB, 0, s>>>(st, ke);
    return 1;
}

// Per-particle log entry (the reference's potE / traj / vel / force buffers,
// EngineUtils.cuh:143-158), written after the step's integration as the
// reference's CompoundIntegrationKernel does (EngineKernels.cuh:399-433): the
// updated position x(t+dt), the potential energy and force of the step's
// evaluation at x(t), and the speed of the stored velocity (velocity Verlet:
// v(t) times the thermostat scale, synchronous with that energy; leapfrog:
// v(t+dt/2)), in original atom order.
__global__ void k_log_frame(DevState st, float4* pos_epot, float4* force_speed) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= st.n_slots) return;
    const int a = st.orig[s];
    if (a < 0) return;
    const float4 v = st.vel[s];
    const float3 F = load_force(st, s);
    pos_epot[a] = make_float4((float)st.px[s], (float)st.py[s], (float)st.pz[s],
                              (float)((double)st.epot[s] * (1.0 / ENERGY_SCALE)));
    force_speed[a] = make_float4(F.x, F.y, F.z, sqrtf(v.x * v.x + v.y * v.y + v.z * v.z));
}

int launch_log_frame(const DevState& st, float4* pos_epot, float4* force_speed, cudaStream_t s) {
    const int TB = 256;
    k_log_frame<<<(st.n_slots + TB - 1) / TB, TB, 0, s>>>(st, pos_epot, force_speed);
    return 1;
}

// State handed in by the caller for atoms that keep their slots, in two steps.
// k_check_state reads the staged input only: word[0] receives the largest
// squared move since the last pair-list build (float bits; it decides on the
// host whether the list still holds), word[1] bit 0 is set when a position is
// not finite, so that the host can refuse the call with the engine untouched,
// and bit 1 when any position differs from the engine's own (a state handed
// back unchanged keeps the list on its usual rebuild cadence).
__global__ void k_check_state(DevState st, int a0, int n, unsigned* word) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float d2 = 0.f;
    bool bad = false, moved = false;
    if (i < n) {
        const int a = a0 + i;
        const int s = st.slot_of[a];
        const double x = st.in_pos[3 * a], y = st.in_pos[3 * a + 1], z = st.in_pos[3 * a + 2];
        bad = !(isfinite(x) && isfinite(y) && isfinite(z));
        moved = x != st.px[s] || y != st.py[s] || z != st.pz[s];
        const float4 r = st.xyz_ref[s];
        const float dx = (float)x - r.x, dy = (float)y - r.y, dz = (float)z - r.z;
        d2 = dx * dx + dy * dy + dz * dz;
        if (!(d2 < 3.0e38f)) d2 = 3.0e38f;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d2 = fmaxf(d2, __shfl_xor_sync(0xffffffffu, d2, o));
    const bool any_bad = __any_sync(0xffffffffu, bad), any_moved = __any_sync(0xffffffffu, moved);
    if ((threadIdx.x & 31) == 0) {
        atomicMax(word, __float_as_uint(d2));
        if (any_bad || any_moved) atomicOr(word + 1, (any_bad ? 1u : 0u) | (any_moved ? 2u : 0u));
    }
}

// ... then k_load_state commits it: positions and velocities replace the slot
// state (previous-step force and minimiser moments restart at zero, as after a
// full rebuild from new input).
__global__ void k_load_state(DevState st, int a0, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int a = a0 + i;
    const int s = st.slot_of[a];
    const double x = st.in_pos[3 * a], y = st.in_pos[3 * a + 1], z = st.in_pos[3 * a + 2];
    st.px[s] = x;
    st.py[s] = y;
    st.pz[s] = z;
    const float4 old = st.xyzq[s];
    st.xyzq[s] = make_float4((float)x, (float)y, (float)z, old.w);
    const float4 v = st.vel[s];
    st.vel[s] = make_float4(st.in_vel[3 * a], st.in_vel[3 * a + 1], st.in_vel[3 * a + 2], v.w);
    st.fprev[s] = make_float4(0.f, 0.f, 0.f, 0.f);
    st.adam_m[s] = make_float4(0.f, 0.f, 0.f, 0.f);
    st.adam_v[s] = make_float4(0.f, 0.f, 0.f, 0.f);
}

int launch_check_state(const DevState& st, int a0, int n, unsigned* word2, cudaStream_t s) {
    const int TB = 256;
    k_check_state<<<(n + TB - 1) / TB, TB, 0, s>>>(st, a0, n, word2);
    return 1;
}

int launch_load_state(const DevState& st, int a0, int n, cudaStream_t s) {
    const int TB = 256;
    k_load_state<<<(n + TB - 1) / TB, TB, 0, s>>>(st, a0, n);
    return 1;
}

int launch_gather_state(const DevState& st, double* pos_out, float* vel_out, cudaStream_t s) {
    const int TB = 256;
    k_gather_state<<<(st.n_atoms + TB - 1) / TB, TB, 0, s>>>(st, pos_out, vel_out);
    return 1;
}

__global__ void k_gather_forces(DevState st, double* f) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= st.n_atoms) return;
    const int s = st.slot_of[a];
    const double inv = 1.0 / FORCE_SCALE;
    f[3 * a] = (double)st.fx[s] * inv;
    f[3 * a + 1] = (double)st.fy[s] * inv;
    f[3 * a + 2] = (double)st.fz[s] * inv;
}

int launch_gather_forces(const DevState& st, double* f_out, cudaStream_t s) {
    const int TB = 256;
    k_gather_forces<<<(st.n_atoms + TB - 1) / TB, TB, 0, s>>>(st, f_out);
    return 1;
}

// fx, fy and fz are one block (fy = fx + n_slots, fz = fy + n_slots)
// Force accumulators at the start of a force evaluation: the external field's
// q E on every atom (EngineKernels.cuh:321-343: the field force joins the
// step's force sum, without potential energy), zero on padding slots.
__global__ void k_field_forces(DevState st) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= st.n_slots) return;
    long long fx = 0, fy = 0, fz = 0;
    if (st.orig[s] >= 0) {
        const SysDesc& sd = st.sys[st.cluster_sys[s / CLUSTER]];
        const float q = st.xyzq[s].w;
        fx = to_fixed(q * sd.efield[0], FORCE_SCALE);
        fy = to_fixed(q * sd.efield[1], FORCE_SCALE);
        fz = to_fixed(q * sd.efield[2], FORCE_SCALE);
    }
    st.fx[s] = fx;
    st.fy[s] = fy;
    st.fz[s] = fz;
}

int launch_zero_forces(const DevState& st, cudaStream_t s) {
    if (st.has_field) {
        k_field_forces<<<(st.n_slots + 255) / 256, 256, 0, s>>>(st);
        return 1;
    }
    cudaMemsetAsync(st.fx, 0, 3 * (size_t)st.n_slots * sizeof(long long), s);
    return 0;  // a memset, not a kernel of this library
}

}  // namespace lima
