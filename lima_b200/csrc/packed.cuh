// packed.cuh — Blackwell packed FP32 arithmetic for the pair kernels.
#pragma once

namespace lima {

// ---------------------------------------------------------------- packed FP32
// Blackwell's packed FP32 instructions ({add,sub,mul,fma}.rn.f32x2, sm_100):
// one instruction computes two lanes of a float pair held in a 64-bit register,
// each rounded exactly like its scalar counterpart.
struct f2p {
    unsigned long long v;
};
__device__ __forceinline__ f2p pk2(float a, float b) {
    f2p r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float2 up2(f2p a) {
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(a.v));
    return r;
}
__device__ __forceinline__ f2p splat2(float a) { return pk2(a, a); }
__device__ __forceinline__ f2p add2(f2p a, f2p b) {
    f2p d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ f2p sub2(f2p a, f2p b) {
    f2p d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ f2p mul2(f2p a, f2p b) {
    f2p d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ f2p fma2(f2p a, f2p b, f2p c) {
    f2p d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return d;
}

}  // namespace lima
