// Common device definitions for the B200 Vamana hot path.
//
// Device data layout (HBM):
//   points : n rows, row stride = round_up(d * sizeof(T), 64) bytes, zero padded
//            (the reference pads rows to 64 B too: include/utils/point_range.h:45-50).
//   graph  : n rows of Rp uint32 (Rp = round_up(R, 4), 16-byte aligned rows);
//            the valid neighbours are a prefix, the rest hold DD_NONE.  This
//            replaces the reference's [deg, nbr...] rows (include/utils/graph.h:
//            126-128): the degree is the length of the valid prefix.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define DD_NONE 0xFFFFFFFFu
#define DD_VBIT 0x80000000u  // "visited" flag carried in frontier ids (ids < 2^31)

// error word bits (OR-ed into a device word; read back by the host)
#define DD_EBAD_ID 0x1u       // a graph row named an id >= n
#define DD_EVIS_CAP 0x2u      // visited list exceeded its capacity
#define DD_ECAND_CAP 0x4u     // a per-query beam width was 0, below k, or above the launch maximum
#define DD_EDEGREE 0x8u       // a row would exceed R (reference aborts: graph.h:61-93)
#define DD_ESEG_CAP 0x10u     // reverse-edge segment exceeded its capacity

enum dd_dtype_e { DD_F32 = 0, DD_I8 = 1, DD_U8 = 2 };
enum dd_metric_e { DD_L2 = 0, DD_MIPS = 1 };

__device__ __forceinline__ void dd_set_error(uint32_t* err, uint32_t bits) {
  if (err) atomicOr(err, bits);
}

// ----------------------------------------------------------------------------
// Exact distances.  Each is computed by ONE thread, in the reference's order:
//   f32 L2   : include/utils/NSGDist.h:113-131 (groups of 4 summed left to
//              right, then added to the running sum; then the 0-3 tail)
//   f32 MIPS : include/utils/mips_point.h:60-66 (sequential sum of products)
//   int L2 / MIPS : exact int32 (include/utils/euclidian_point.h:44-60,
//              mips_point.h:44-58), returned as float (round to nearest).
// The _rn intrinsics keep nvcc from contracting into FMA, so float results are
// bit-identical to the reference's x86-64 scalar build.
// `a` may live in shared or global memory, `b` in global memory; both rows are
// 16-byte aligned and zero padded to a multiple of 16 bytes.
// ----------------------------------------------------------------------------
template <int DT, int MT>
struct Dist;

template <>
struct Dist<DD_F32, DD_L2> {
  static __device__ __forceinline__ float eval(const void* av, const void* bv, uint32_t d) {
    const float* a = (const float*)av;
    const float4* b4 = (const float4*)bv;
    float r = 0.f;
    uint32_t i = 0;
#pragma unroll 8
    for (; i + 3 < d; i += 4) {
      float4 x = *(const float4*)(a + i);
      float4 y = __ldg(b4 + (i >> 2));
      float d0 = __fsub_rn(x.x, y.x), d1 = __fsub_rn(x.y, y.y);
      float d2 = __fsub_rn(x.z, y.z), d3 = __fsub_rn(x.w, y.w);
      float s = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(d0, d0), __fmul_rn(d1, d1)),
                                    __fmul_rn(d2, d2)),
                          __fmul_rn(d3, d3));
      r = __fadd_rn(r, s);
    }
    const float* b = (const float*)bv;
    for (; i < d; i++) {
      float d0 = __fsub_rn(a[i], __ldg(b + i));
      r = __fadd_rn(r, __fmul_rn(d0, d0));
    }
    return r;
  }
};

template <>
struct Dist<DD_F32, DD_MIPS> {
  static __device__ __forceinline__ float eval(const void* av, const void* bv, uint32_t d) {
    const float* a = (const float*)av;
    const float4* b4 = (const float4*)bv;
    float r = 0.f;
    uint32_t i = 0;
#pragma unroll 8
    for (; i + 3 < d; i += 4) {
      float4 x = *(const float4*)(a + i);
      float4 y = __ldg(b4 + (i >> 2));
      r = __fadd_rn(r, __fmul_rn(x.x, y.x));
      r = __fadd_rn(r, __fmul_rn(x.y, y.y));
      r = __fadd_rn(r, __fmul_rn(x.z, y.z));
      r = __fadd_rn(r, __fmul_rn(x.w, y.w));
    }
    const float* b = (const float*)bv;
    for (; i < d; i++) r = __fadd_rn(r, __fmul_rn(a[i], __ldg(b + i)));
    return -r;
  }
};

// integer forms: 16 bytes per step, zero padding contributes nothing
template <int DT>
__device__ __forceinline__ uint32_t absdiff4(uint32_t x, uint32_t y) {
  if (DT == DD_U8) return __vabsdiffu4(x, y);
  return __vabsdiffs4(x, y);  // |a-b| <= 255 fits the unsigned byte lane
}

template <int DT>
struct DistIntL2 {
  static __device__ __forceinline__ float eval(const void* av, const void* bv, uint32_t d) {
    const uint4* a = (const uint4*)av;
    const uint4* b = (const uint4*)bv;
    uint32_t acc = 0;
    uint32_t nv = (d + 15) >> 4;
#pragma unroll 8
    for (uint32_t i = 0; i < nv; i++) {
      uint4 x = a[i];
      uint4 y = __ldg(b + i);
      uint32_t t;
      t = absdiff4<DT>(x.x, y.x); acc = __dp4a(t, t, acc);
      t = absdiff4<DT>(x.y, y.y); acc = __dp4a(t, t, acc);
      t = absdiff4<DT>(x.z, y.z); acc = __dp4a(t, t, acc);
      t = absdiff4<DT>(x.w, y.w); acc = __dp4a(t, t, acc);
    }
    return __int2float_rn((int)acc);
  }
};

template <int DT>
struct DistIntIP {
  static __device__ __forceinline__ float eval(const void* av, const void* bv, uint32_t d) {
    const uint4* a = (const uint4*)av;
    const uint4* b = (const uint4*)bv;
    int acc = 0;
    uint32_t nv = (d + 15) >> 4;
#pragma unroll 8
    for (uint32_t i = 0; i < nv; i++) {
      uint4 x = a[i];
      uint4 y = __ldg(b + i);
      if (DT == DD_U8) {
        acc = (int)__dp4a(x.x, y.x, (uint32_t)acc);
        acc = (int)__dp4a(x.y, y.y, (uint32_t)acc);
        acc = (int)__dp4a(x.z, y.z, (uint32_t)acc);
        acc = (int)__dp4a(x.w, y.w, (uint32_t)acc);
      } else {
        acc = __dp4a((int)x.x, (int)y.x, acc);
        acc = __dp4a((int)x.y, (int)y.y, acc);
        acc = __dp4a((int)x.z, (int)y.z, acc);
        acc = __dp4a((int)x.w, (int)y.w, acc);
      }
    }
    return -__int2float_rn(acc);
  }
};

// exact integer value of the integer forms (ground truth)
template <int DT, int MT>
struct DistIntRaw {
  static __device__ __forceinline__ int eval(const void* av, const void* bv, uint32_t d) {
    const uint4* a = (const uint4*)av;
    const uint4* b = (const uint4*)bv;
    uint32_t nv = (d + 15) >> 4;
    if (MT == DD_L2) {
      uint32_t acc = 0;
      for (uint32_t i = 0; i < nv; i++) {
        uint4 x = a[i], y = __ldg(b + i);
        uint32_t t;
        t = absdiff4<DT>(x.x, y.x); acc = __dp4a(t, t, acc);
        t = absdiff4<DT>(x.y, y.y); acc = __dp4a(t, t, acc);
        t = absdiff4<DT>(x.z, y.z); acc = __dp4a(t, t, acc);
        t = absdiff4<DT>(x.w, y.w); acc = __dp4a(t, t, acc);
      }
      return (int)acc;
    }
    int acc = 0;
    for (uint32_t i = 0; i < nv; i++) {
      uint4 x = a[i], y = __ldg(b + i);
      if (DT == DD_U8) {
        acc = (int)__dp4a(x.x, y.x, (uint32_t)acc);
        acc = (int)__dp4a(x.y, y.y, (uint32_t)acc);
        acc = (int)__dp4a(x.z, y.z, (uint32_t)acc);
        acc = (int)__dp4a(x.w, y.w, (uint32_t)acc);
      } else {
        acc = __dp4a((int)x.x, (int)y.x, acc);
        acc = __dp4a((int)x.y, (int)y.y, acc);
        acc = __dp4a((int)x.z, (int)y.z, acc);
        acc = __dp4a((int)x.w, (int)y.w, acc);
      }
    }
    return -acc;
  }
};

template <> struct Dist<DD_I8, DD_L2> : DistIntL2<DD_I8> {};
template <> struct Dist<DD_U8, DD_L2> : DistIntL2<DD_U8> {};
template <> struct Dist<DD_I8, DD_MIPS> : DistIntIP<DD_I8> {};
template <> struct Dist<DD_U8, DD_MIPS> : DistIntIP<DD_U8> {};

// size of one element
template <int DT>
struct ElemSize { static constexpr int v = (DT == DD_F32) ? 4 : 1; };

// Distance from the query `q` (16-byte words, shared memory) to `row` computed
// by a group of G lanes (G = 1, 2, 4 or 8, warp-uniform; `sub` = lane index in
// the group).  Integer data: each lane sums the words sub, sub+G, ... and the
// group adds the partial sums (exact integers, so any grouping gives the
// reference's value).  Float data must keep the reference's summation order:
// G must be 1 and the lane runs Dist::eval.  Every lane of the warp must call
// it (the group reduction shuffles); lanes with act == false return 0.
// NB: 16-byte words a lane loads per batch (its registers in flight).
template <int DT, int MT, int NB = 8>
__device__ __forceinline__ float dist_group(const uint4* q, const uint8_t* row, uint32_t d,
                                            uint32_t sub, uint32_t G, bool act) {
  if (DT == DD_F32) return act ? Dist<DT, MT>::eval(q, row, d) : 0.f;
  const uint32_t nv = (d + 15) >> 4;
  const uint4* r4 = (const uint4*)row;
  uint32_t acc = 0;
  for (uint32_t w0 = sub; w0 < nv; w0 += NB * G) {
    uint4 y[NB];
#pragma unroll
    for (int i = 0; i < NB; i++) {
      const uint32_t w = w0 + (uint32_t)i * G;
      y[i] = (act && w < nv) ? __ldg(r4 + w) : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int i = 0; i < NB; i++) {
      const uint32_t w = w0 + (uint32_t)i * G;
      if (w < nv) {
        const uint4 x = q[w];
        if (MT == DD_L2) {
          uint32_t s;
          s = absdiff4<DT>(x.x, y[i].x); acc = __dp4a(s, s, acc);
          s = absdiff4<DT>(x.y, y[i].y); acc = __dp4a(s, s, acc);
          s = absdiff4<DT>(x.z, y[i].z); acc = __dp4a(s, s, acc);
          s = absdiff4<DT>(x.w, y[i].w); acc = __dp4a(s, s, acc);
        } else if (DT == DD_U8) {
          acc = __dp4a(x.x, y[i].x, acc); acc = __dp4a(x.y, y[i].y, acc);
          acc = __dp4a(x.z, y[i].z, acc); acc = __dp4a(x.w, y[i].w, acc);
        } else {
          int v = (int)acc;
          v = __dp4a((int)x.x, (int)y[i].x, v); v = __dp4a((int)x.y, (int)y[i].y, v);
          v = __dp4a((int)x.z, (int)y[i].z, v); v = __dp4a((int)x.w, (int)y[i].w, v);
          acc = (uint32_t)v;
        }
      }
    }
  }
  // wrap-around uint32 adds give the exact int32 total
  for (uint32_t o = 1; o < G; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (!act) return 0.f;
  return MT == DD_L2 ? __int2float_rn((int)acc) : -__int2float_rn((int)acc);
}

// splitmix64 finaliser: the reference's lossy "seen" filter hashes ids with it
// (include/utils/beamSearch.h:66-73, include/parlay/utilities.h:145-150).
__device__ __forceinline__ uint64_t dd_hash64(uint64_t x) {
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

// (dist, id) order of the beam: include/utils/beamSearch.h:59-61
__device__ __forceinline__ bool pair_less(float da, uint32_t ia, float db, uint32_t ib) {
  return da < db || (da == db && ia < ib);
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }

// CTA-wide exclusive scan (all threads of the block call it; sh: 32 words)
__device__ __forceinline__ uint32_t cta_scan_excl(uint32_t v, uint32_t* total, uint32_t* sh) {
  const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    uint32_t s = lane < nw ? sh[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= (uint32_t)o) s += y;
    }
    if (lane < nw) sh[lane] = s;
  }
  __syncthreads();
  uint32_t wb = w ? sh[w - 1] : 0;
  *total = sh[nw - 1];
  __syncthreads();
  return wb + x - v;
}
