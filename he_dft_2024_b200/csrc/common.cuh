// common.cuh -- shared device helpers for the sm_100a mean-field / time-step kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#define HE_HD __host__ __device__ __forceinline__
#define HE_D __device__ __forceinline__

namespace he {

// ---- complex binary64 arithmetic on double2 (re, im) ------------------------------------------
HE_HD double2 c2(double re, double im) { return make_double2(re, im); }
HE_HD double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
HE_HD double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
HE_HD double2 cscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
HE_HD double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
HE_HD double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
HE_HD double2 cmul_conj_if(double2 a, double2 w, bool conj_w) {
  double wy = conj_w ? -w.y : w.y;
  return make_double2(a.x * w.x - a.y * wy, a.x * wy + a.y * w.x);
}
HE_HD double cnorm2(double2 a) { return a.x * a.x + a.y * a.y; }
// -i * a
HE_HD double2 cmi(double2 a) { return make_double2(a.y, -a.x); }
// +i * a
HE_HD double2 cpi(double2 a) { return make_double2(-a.y, a.x); }

// ---- complex binary32 (the mixed-precision FFT chain) -------------------------------------------
HE_HD float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
HE_HD float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
HE_HD float2 cscale(float s, float2 a) { return make_float2(s * a.x, s * a.y); }
HE_HD float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
HE_HD float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
HE_HD float2 cmul_conj_if(float2 a, float2 w, bool conj_w) {
  float wy = conj_w ? -w.y : w.y;
  return make_float2(a.x * w.x - a.y * wy, a.x * wy + a.y * w.x);
}
HE_HD float2 cmi(float2 a) { return make_float2(a.y, -a.x); }
HE_HD float2 cpi(float2 a) { return make_float2(-a.y, a.x); }

// Complex type of a real type: Cx<double>::T = double2, Cx<float>::T = float2.
template <typename R> struct Cx;
template <> struct Cx<double> {
  using T = double2;
  static HE_HD double2 make(double a, double b) { return make_double2(a, b); }
};
template <> struct Cx<float> {
  using T = float2;
  static HE_HD float2 make(float a, float b) { return make_float2(a, b); }
};

// Generic helpers so stencil code can be written once for real and complex fields.
HE_HD double zero_of(double) { return 0.0; }
HE_HD double2 zero_of(double2) { return make_double2(0.0, 0.0); }
HE_HD double axpy(double w, double f, double acc) { return acc + w * f; }
HE_HD double2 axpy(double w, double2 f, double2 acc) {
  return make_double2(acc.x + w * f.x, acc.y + w * f.y);
}
HE_HD double neg_if(double v, bool n) { return n ? -v : v; }
HE_HD double2 neg_if(double2 v, bool n) { return n ? make_double2(-v.x, -v.y) : v; }
HE_HD float zero_of(float) { return 0.0f; }
HE_HD float2 zero_of(float2) { return make_float2(0.0f, 0.0f); }
HE_HD float axpy(float w, float f, float acc) { return fmaf(w, f, acc); }
HE_HD float2 axpy(float w, float2 f, float2 acc) {
  return make_float2(fmaf(w, f.x, acc.x), fmaf(w, f.y, acc.y));
}
HE_HD float neg_if(float v, bool n) { return n ? -v : v; }
HE_HD float2 neg_if(float2 v, bool n) { return n ? make_float2(-v.x, -v.y) : v; }
HE_HD float cnorm2(float2 a) { return a.x * a.x + a.y * a.y; }

// Real type of a stencil field type (double for double/double2, float for float/float2): the
// operand fields of a stencil consumer have the precision of the field it differentiates.
template <typename T> struct RealOf { using R = double; using Z = double2; };
template <> struct RealOf<float> { using R = float; using Z = float2; };
template <> struct RealOf<float2> { using R = float; using Z = float2; };

// ---- compensated binary32 pairs (hi, lo): value hi + lo, |lo| <= ulp(hi)/2 -----------------------
// The mixed path keeps psi and its history as such pairs (about 48 significant bits) and updates
// them with error-free transformations; the _rn intrinsics keep the compiler from contracting or
// reassociating the steps.
struct HL {
  float hi, lo;
};
// Knuth's TwoSum: s + e = a + b exactly.
HE_D void two_sum(float a, float b, float& s, float& e) {
  s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}
// Dekker's FastTwoSum (|a| >= |b| or a = 0): s + e = a + b exactly.
HE_D HL fast_two_sum(float a, float b) {
  const float s = __fadd_rn(a, b);
  return HL{s, __fsub_rn(b, __fsub_rn(s, a))};
}
// (hi, lo) + b
HE_D HL hl_add(HL a, float b) {
  float s, e;
  two_sum(a.hi, b, s, e);
  return fast_two_sum(s, __fadd_rn(e, a.lo));
}
// (hi, lo) + (hi, lo)
HE_D HL hl_add(HL a, HL b) {
  float s, e;
  two_sum(a.hi, b.hi, s, e);
  return fast_two_sum(s, __fadd_rn(e, __fadd_rn(a.lo, b.lo)));
}
HE_D HL hl_neg(HL a) { return HL{-a.hi, -a.lo}; }
// c * (hi, lo) with a binary32 constant c (the product hi*c split exactly by an fma)
HE_D HL hl_mul(float c, HL a) {
  const float p = __fmul_rn(c, a.hi);
  const float e = __fmaf_rn(c, a.lo, __fmaf_rn(c, a.hi, -p));
  return fast_two_sum(p, e);
}
// binary64 <-> pair (host and device)
HE_HD HL hl_from(double v) {
  const float h = (float)v;
  return HL{h, (float)(v - (double)h)};
}
HE_HD double hl_value(HL a) { return (double)a.hi + (double)a.lo; }

// Asynchronous global -> shared copy of one element (cp.async, zero fill when src_bytes = 0).
template <typename T>
HE_D void cp_async_elem(T* dst_smem, const T* src, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(dst_smem);
  const int nbytes = valid ? (int)sizeof(T) : 0;
  if constexpr (sizeof(T) == 16) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(src),
                 "r"(nbytes));
  } else if constexpr (sizeof(T) == 8) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(src),
                 "r"(nbytes));
  } else {
    static_assert(sizeof(T) == 4, "cp.async copies 4, 8 or 16 bytes");
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(src),
                 "r"(nbytes));
  }
}
HE_D void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
HE_D void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// 16 bytes global -> shared (both addresses 16-byte aligned).
HE_D void cp_async16(void* dst_smem, const void* src) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(src));
}
// A contiguous byte range global -> shared in 16-byte pieces spread over the CTA's threads
// (bytes a multiple of 16, both ends 16-byte aligned).
HE_D void cp_async_range(void* dst_smem, const void* src, long bytes, int tid, int nthr) {
  char* d = static_cast<char*>(dst_smem);
  const char* g = static_cast<const char*>(src);
  for (long o = 16L * tid; o < bytes; o += 16L * nthr) cp_async16(d + o, g + o);
}

// ---- programmatic dependent launch ------------------------------------------------------------
// The FFT passes of the step chain are launched with programmatic stream serialisation: a pass
// may be scheduled while its predecessor in the stream drains, and waits here, before its first
// access to global memory, until the predecessor has completed and its writes are visible.
// Without the launch attribute both instructions are no-ops.  The trigger lets the successor be
// scheduled once every CTA of this kernel has started.
HE_D void pdl_wait_and_trigger() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

// ---- members of a context group ----------------------------------------------------------------
// A group (he_ctx_group) advances several contexts of identical geometry with one launch per
// kernel: the leader's launches carry a grid dimension over the members, and every CTA of member
// m maps each device pointer of its arguments -- all of them the leader's buffers -- to member
// m's corresponding buffer through this table: the leader's buffer starts (ascending) and sizes,
// then per member the starts of its buffers in the same order.  A pointer inside no leader buffer
// is returned unchanged, and so is every pointer of member 0 (the leader itself, and every
// context that is not in a group: nmem = 1, no table).
struct MemberMap {
  const unsigned long long* tab;  // [nbuf] leader starts, [nbuf] sizes, [nmem][nbuf] member starts
  int nbuf, nmem;
  template <class T>
  HE_D T* operator()(T* p, int m) const {
    if (m == 0 || p == nullptr || nbuf == 0) return p;
    const unsigned long long a = reinterpret_cast<unsigned long long>(p);
    int lo = 0, hi = nbuf - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(tab + mid) <= a) lo = mid;
      else hi = mid - 1;
    }
    const unsigned long long b = __ldg(tab + lo);
    if (a < b || a >= b + __ldg(tab + nbuf + lo)) return p;
    return reinterpret_cast<T*>(__ldg(tab + 2 * nbuf + (size_t)m * nbuf + lo) + (a - b));
  }
};

// Pointer p of member m: mapped through mm in the group instantiation (G) of a kernel, returned
// unchanged otherwise.
template <bool G, class T>
HE_D T* on_member(const MemberMap& mm, T* p, int m) {
  if constexpr (G) return mm(p, m);
  else return p;
}

// The heavy kernel templates (stencils, FFT passes) are compiled in their own translation units,
// which define HE_KERNEL_TU and instantiate the kernels the host code launches; the host
// translation unit sees their declarations only.

// ---- block reduction of NV doubles (fixed order => deterministic) ------------------------------
template <int NV>
__device__ void block_reduce_store(double (&v)[NV], double* __restrict__ out) {
  __shared__ double red[32][NV > 0 ? NV : 1];
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthr = blockDim.x * blockDim.y * blockDim.z;
  const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double s = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) red[warp][k] = s;
  }
  __syncthreads();
  if (tid == 0) {
    const int nw = (nthr + 31) >> 5;
    for (int k = 0; k < NV; ++k) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += red[w][k];
      out[k] = s;
    }
  }
}

}  // namespace he
