// gb_device.cuh -- device building blocks of the hash groupby engine:
// key packing, hashing, open-addressing find-or-insert (global and shared
// memory), accumulator updates/merges and output finalisation.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "gb_plan.h"

namespace gb {

constexpr uint64_t kEmpty = ~0ull;   // key word of an empty slot
constexpr uint32_t kNoRow32 = 0xFFFFFFFFu;

// ---------------------------------------------------------------------------
// element loads
__device__ __forceinline__ bool bit_valid(const uint32_t* m, int64_t i)
{
  return m == nullptr || ((__ldg(m + (i >> 5)) >> (i & 31)) & 1u);
}

__device__ __forceinline__ uint64_t load_bits(const void* base, int64_t i, int width)
{
  switch (width) {
    case 1: return __ldg((const uint8_t*)base + i);
    case 2: return __ldg((const uint16_t*)base + i);
    case 4: return __ldg((const uint32_t*)base + i);
    default: return __ldg((const unsigned long long*)base + i);
  }
}

__device__ __forceinline__ int64_t sign_extend(uint64_t bits, int width)
{
  switch (width) {
    case 1: return (int8_t)bits;
    case 2: return (int16_t)bits;
    case 4: return (int32_t)bits;
    default: return (int64_t)bits;
  }
}

// normalised key bits: all NaNs one value, -0.0 == +0.0, bool -> 0/1
// (libcudf hashes and compares keys this way:
//  cpp/include/cudf/hashing/detail/murmurhash3_x86_32.cuh:66-68)
__device__ __forceinline__ uint64_t norm_key_bits(const KeyCol& c, uint64_t b)
{
  if (c.cat == CAT_F32) {
    float f = __uint_as_float((uint32_t)b);
    if (f != f) return 0x7FC00000u;
    if (f == 0.0f) return 0;
    return b;
  }
  if (c.cat == CAT_F64) {
    double d = __longlong_as_double((long long)b);
    if (d != d) return 0x7FF8000000000000ull;
    if (d == 0.0) return 0;
    return b;
  }
  if (c.cat == CAT_BOOL) return b != 0;
  return b;
}
__device__ __forceinline__ uint64_t key_bits(const KeyCol& c, int64_t r)
{
  return norm_key_bits(c, load_bits(c.data, r, c.width));
}

// Packs the key tuple of a row into one or two 64-bit words.  Returns false
// when null_policy::EXCLUDE drops the row (a null in any key column;
// cpp/src/groupby/hash/groupby.cu:482-485).
__device__ __forceinline__ bool pack_key(const Plan& P, int64_t row, uint64_t& w0, uint64_t& w1)
{
  w0 = 0;
  w1 = 0;
#pragma unroll 1
  for (int k = 0; k < P.num_keys; ++k) {
    const KeyCol& c = P.keys[k];
    int64_t r = row + c.offset;
    if (!bit_valid(c.mask, r)) {
      if (!P.include_nulls) return false;
      uint64_t nb = 1ull << c.null_shift;
      if (c.null_word == 0) w0 |= nb; else w1 |= nb;
      continue;
    }
    uint64_t v = key_bits(c, r) << c.shift;
    if (c.word == 0) w0 |= v; else w1 |= v;
  }
  return true;
}

// MurmurHash3 fmix64 finaliser (Appleby, public domain)
__device__ __forceinline__ uint64_t fmix64(uint64_t k)
{
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return k;
}
__device__ __forceinline__ uint64_t hash_key(uint64_t w0, uint64_t w1, int words)
{
  return words == 1 ? fmix64(w0) : fmix64(w0 ^ fmix64(w1 + 0x9E3779B97F4A7C15ull));
}

// 16-byte volatile load (generic address: global or shared)
__device__ __forceinline__ ulonglong2 vload2(const void* p)
{
  ulonglong2 r;
  asm volatile("ld.volatile.v2.u64 {%0, %1}, [%2];" : "=l"(r.x), "=l"(r.y) : "l"(p) : "memory");
  return r;
}

// ---------------------------------------------------------------------------
// find-or-insert.  Slot i starts at T + i*stride with its key word(s).
// Returns the slot index, `special` (= capacity) for the all-ones key of a
// one-word table, or -1 when the table is full (bounded: at most capacity
// probes).  `inserted` is set when this call claimed the slot.
__device__ __forceinline__ int64_t find_or_insert1(uint8_t* T, int stride, uint64_t cap_mask,
                                                   uint64_t key, uint64_t h, int max_probes,
                                                   bool& inserted)
{
  inserted = false;
  if (key == kEmpty) return (int64_t)cap_mask + 1;
  uint64_t i = h & cap_mask;
  for (int p = 0; p < max_probes; ++p) {
    unsigned long long* kp = (unsigned long long*)(T + i * (uint64_t)stride);
    uint64_t cur = *(volatile unsigned long long*)kp;
    if (cur == key) return (int64_t)i;
    if (cur == kEmpty) {
      uint64_t old = atomicCAS(kp, kEmpty, key);
      if (old == kEmpty) { inserted = true; return (int64_t)i; }
      if (old == key) return (int64_t)i;
    }
    i = (i + 1) & cap_mask;
  }
  return -1;
}

// Two-word keys keep the top bit of word 1 clear (at most 127 key bits), so a
// slot whose word 1 has that bit set is empty or still being written.  Keys are
// claimed with one 128-bit CAS; a read that could be torn is repeated with the
// CAS (compare = empty) to get the untorn contents.
__device__ __forceinline__ int64_t find_or_insert2(uint8_t* T, int stride, uint64_t cap_mask,
                                                   uint64_t k0, uint64_t k1, uint64_t h,
                                                   int max_probes, bool& inserted)
{
  inserted = false;
  uint64_t i = h & cap_mask;
  unsigned __int128 want = ((unsigned __int128)k1 << 64) | k0;
  const unsigned __int128 empty = ~(unsigned __int128)0;
  for (int p = 0; p < max_probes; ++p) {
    unsigned __int128* kp = (unsigned __int128*)(T + i * (uint64_t)stride);
    ulonglong2 cur = vload2(kp);
    if (cur.x == k0 && cur.y == k1 && k0 != kEmpty) return (int64_t)i;
    if ((cur.y >> 63) || cur.x == kEmpty) {
      unsigned __int128 old = atomicCAS(kp, empty, want);
      if (old == empty) { inserted = true; return (int64_t)i; }
      if (old == want) return (int64_t)i;
    }
    i = (i + 1) & cap_mask;
  }
  return -1;
}

// lookup only (second pass); -1 when absent
__device__ __forceinline__ int64_t find1(const uint8_t* T, int stride, uint64_t cap_mask,
                                         uint64_t key, uint64_t h)
{
  if (key == kEmpty) return (int64_t)cap_mask + 1;
  uint64_t i = h & cap_mask;
  for (uint64_t p = 0; p <= cap_mask; ++p) {
    uint64_t cur = *(const unsigned long long*)(T + i * (uint64_t)stride);
    if (cur == key) return (int64_t)i;
    if (cur == kEmpty) return -1;
    i = (i + 1) & cap_mask;
  }
  return -1;
}
__device__ __forceinline__ int64_t find2(const uint8_t* T, int stride, uint64_t cap_mask,
                                         uint64_t k0, uint64_t k1, uint64_t h)
{
  uint64_t i = h & cap_mask;
  for (uint64_t p = 0; p <= cap_mask; ++p) {
    ulonglong2 cur = *(const ulonglong2*)(T + i * (uint64_t)stride);
    if (cur.x == k0 && cur.y == k1) return (int64_t)i;
    if (cur.y >> 63) return -1;
    i = (i + 1) & cap_mask;
  }
  return -1;
}

// ---------------------------------------------------------------------------
// order-preserving unsigned encodings for MIN/MAX/ARG*
__device__ __forceinline__ uint32_t ord32_f(float f, bool for_min)
{
  // +qNaN encodes just above +inf (MIN ignores it), -qNaN just below -inf
  if (f != f) return for_min ? 0xFFC00000u : 0x003FFFFFu;
  uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float dec32_f(uint32_t e)
{
  uint32_t b = (e & 0x80000000u) ? (e & 0x7FFFFFFFu) : ~e;
  return __uint_as_float(b);
}
__device__ __forceinline__ uint64_t ord64_f(double d, bool for_min)
{
  if (d != d) return for_min ? 0xFFF8000000000000ull : 0x0007FFFFFFFFFFFFull;
  uint64_t b = (uint64_t)__double_as_longlong(d);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dec64_f(uint64_t e)
{
  uint64_t b = (e >> 63) ? (e & 0x7FFFFFFFFFFFFFFFull) : ~e;
  return __longlong_as_double((long long)b);
}

// Loaded value of one row of a value column.
struct Elem {
  uint64_t bits;   // raw bits (zero-extended)
  int64_t i;       // integral value (sign- or zero-extended; bool as 0/1)
  double d;        // floating value (f32 widened)
  float f;
};

__device__ __forceinline__ Elem load_elem(const ValCol& c, int64_t r)
{
  Elem e;
  e.bits = load_bits(c.data, r, c.width);
  switch (c.cat) {
    case CAT_SIGNED: e.i = sign_extend(e.bits, c.width); break;
    case CAT_BOOL: e.i = e.bits != 0; break;
    case CAT_UNSIGNED: e.i = (int64_t)e.bits; break;
    case CAT_F32: e.f = __uint_as_float((uint32_t)e.bits); e.d = e.f; break;
    default: e.d = __longlong_as_double((long long)e.bits); break;
  }
  return e;
}

__device__ __forceinline__ uint32_t ord32(const ValCol& c, const Elem& e, bool for_min)
{
  switch (c.cat) {
    case CAT_F32: return ord32_f(e.f, for_min);
    case CAT_UNSIGNED: return (uint32_t)e.bits;
    case CAT_BOOL: return (uint32_t)e.i;
    default: return (uint32_t)(int32_t)e.i ^ 0x80000000u;
  }
}
__device__ __forceinline__ uint64_t ord64(const ValCol& c, const Elem& e, bool for_min)
{
  switch (c.cat) {
    case CAT_F64: return ord64_f(e.d, for_min);
    case CAT_UNSIGNED: return e.bits;
    default: return (uint64_t)e.i ^ 0x8000000000000000ull;
  }
}

template <typename T>
__device__ __forceinline__ T vload(const void* p)
{
  return *(const volatile T*)p;
}

// 64-bit CAS-loop product (libcudf's atomic_mul is a CAS loop as well:
// cpp/include/cudf/detail/utilities/device_atomics.cuh:132-153)
__device__ __forceinline__ void atomic_mul_i64(unsigned long long* p, uint64_t x)
{
  unsigned long long old = vload<unsigned long long>(p), assumed;
  do {
    assumed = old;
    old = atomicCAS(p, assumed, assumed * x);
  } while (old != assumed);
}
__device__ __forceinline__ void atomic_mul_f64(unsigned long long* p, double x)
{
  unsigned long long old = vload<unsigned long long>(p), assumed;
  do {
    assumed = old;
    double v = __longlong_as_double((long long)assumed) * x;
    old = atomicCAS(p, assumed, (unsigned long long)__double_as_longlong(v));
  } while (old != assumed);
}
__device__ __forceinline__ void atomic_mul_f32(unsigned int* p, float x)
{
  unsigned int old = vload<unsigned int>(p), assumed;
  do {
    assumed = old;
    float v = __uint_as_float(assumed) * x;
    old = atomicCAS(p, assumed, __float_as_uint(v));
  } while (old != assumed);
}

// (value,row) comparison through the column for 64-bit ARGMIN/ARGMAX.
__device__ __forceinline__ bool arg_better(const ValCol& c, uint64_t enc_new, uint32_t row_new,
                                           uint64_t row_old, bool is_min)
{
  Elem o = load_elem(c, (int64_t)row_old + c.offset);
  uint64_t eo = ord64(c, o, is_min);
  if (enc_new != eo) return is_min ? enc_new < eo : enc_new > eo;
  return row_new < row_old;
}
__device__ __forceinline__ void atomic_arg_r64(unsigned long long* p, const ValCol& c,
                                               uint64_t enc, uint32_t row, bool is_min)
{
  unsigned long long old = vload<unsigned long long>(p);
  for (;;) {
    if (old != kEmpty && !arg_better(c, enc, row, old, is_min)) return;
    unsigned long long prev = atomicCAS(p, old, (unsigned long long)row);
    if (prev == old) return;
    old = prev;
  }
}

// Applies one valid element to the accumulators [a0, a1) of a slot.
// Works on global and shared slots alike (generic addressing).
__device__ __forceinline__ void apply_elem(const Plan& P, const ValCol& c, int a0, int a1,
                                           uint8_t* slot, const Elem& e, uint32_t row)
{
#pragma unroll 1
  for (int a = a0; a < a1; ++a) {
    const Acc A = P.accs[a];
    uint8_t* p = slot + A.off;
    switch (A.op) {
      case OP_SUM_I64: atomicAdd((unsigned long long*)p, (unsigned long long)e.i); break;
      case OP_SUM_I32: atomicAdd((unsigned int*)p, (unsigned int)e.i); break;
      case OP_SUM_F32: atomicAdd((float*)p, e.f); break;
      case OP_SUM_F64: atomicAdd((double*)p, e.d); break;
      case OP_MIN_U32: {
        uint32_t v = ord32(c, e, true);
        if (v < vload<uint32_t>(p)) atomicMin((unsigned int*)p, v);
        break;
      }
      case OP_MAX_U32: {
        uint32_t v = ord32(c, e, false);
        if (v > vload<uint32_t>(p)) atomicMax((unsigned int*)p, v);
        break;
      }
      case OP_MIN_U64: {
        uint64_t v = ord64(c, e, true);
        if (v < vload<unsigned long long>(p)) atomicMin((unsigned long long*)p, v);
        break;
      }
      case OP_MAX_U64: {
        uint64_t v = ord64(c, e, false);
        if (v > vload<unsigned long long>(p)) atomicMax((unsigned long long*)p, v);
        break;
      }
      case OP_SQ_I64: atomicAdd((unsigned long long*)p, (unsigned long long)e.i * (unsigned long long)e.i); break;
      case OP_SQ_F32: atomicAdd((float*)p, e.f * e.f); break;
      case OP_SQ_F64: atomicAdd((double*)p, e.d * e.d); break;
      case OP_PROD_I64: atomic_mul_i64((unsigned long long*)p, (uint64_t)e.i); break;
      case OP_PROD_F32: atomic_mul_f32((unsigned int*)p, e.f); break;
      case OP_PROD_F64: atomic_mul_f64((unsigned long long*)p, e.d); break;
      case OP_ARGMIN_P32: {
        uint64_t v = ((uint64_t)ord32(c, e, true) << 32) | row;
        if (v < vload<unsigned long long>(p)) atomicMin((unsigned long long*)p, v);
        break;
      }
      case OP_ARGMAX_P32: {
        uint64_t v = ((uint64_t)ord32(c, e, false) << 32) | (uint32_t)~row;
        if (v > vload<unsigned long long>(p)) atomicMax((unsigned long long*)p, v);
        break;
      }
      case OP_ARGMIN_R64: atomic_arg_r64((unsigned long long*)p, c, ord64(c, e, true), row, true); break;
      case OP_ARGMAX_R64: atomic_arg_r64((unsigned long long*)p, c, ord64(c, e, false), row, false); break;
      default: break;
    }
  }
}

// Merges accumulator a of slot `src` into slot `dst` (dst: global).
__device__ __forceinline__ void merge_acc(const Plan& P, const Acc& A, uint8_t* dst, const uint8_t* src)
{
  uint8_t* d = dst + A.off;
  const uint8_t* s = src + A.off;
  switch (A.op) {
    case OP_NULLS: { uint32_t v = *(const uint32_t*)s; if (v) atomicAdd((unsigned int*)d, v); break; }
    case OP_SUM_I64: case OP_SQ_I64: {
      unsigned long long v = *(const unsigned long long*)s;
      if (v) atomicAdd((unsigned long long*)d, v);
      break;
    }
    case OP_SUM_I32: { uint32_t v = *(const uint32_t*)s; if (v) atomicAdd((unsigned int*)d, v); break; }
    case OP_SUM_F32: case OP_SQ_F32: { float v = *(const float*)s; if (v != 0.0f) atomicAdd((float*)d, v); break; }
    case OP_SUM_F64: case OP_SQ_F64: { double v = *(const double*)s; if (v != 0.0) atomicAdd((double*)d, v); break; }
    case OP_MIN_U32: { uint32_t v = *(const uint32_t*)s; if (v != 0xFFFFFFFFu) atomicMin((unsigned int*)d, v); break; }
    case OP_MAX_U32: { uint32_t v = *(const uint32_t*)s; if (v != 0u) atomicMax((unsigned int*)d, v); break; }
    case OP_MIN_U64: case OP_ARGMIN_P32: {
      unsigned long long v = *(const unsigned long long*)s;
      if (v != kEmpty) atomicMin((unsigned long long*)d, v);
      break;
    }
    case OP_MAX_U64: case OP_ARGMAX_P32: {
      unsigned long long v = *(const unsigned long long*)s;
      if (v != 0ull) atomicMax((unsigned long long*)d, v);
      break;
    }
    case OP_PROD_I64: { uint64_t v = *(const uint64_t*)s; if (v != 1) atomic_mul_i64((unsigned long long*)d, v); break; }
    case OP_PROD_F32: { float v = *(const float*)s; if (v != 1.0f) atomic_mul_f32((unsigned int*)d, v); break; }
    case OP_PROD_F64: { double v = *(const double*)s; if (v != 1.0) atomic_mul_f64((unsigned long long*)d, v); break; }
    case OP_ARGMIN_R64: case OP_ARGMAX_R64: {
      unsigned long long r = *(const unsigned long long*)s;
      if (r != kEmpty) {
        const ValCol& c = P.vals[A.col];
        Elem e = load_elem(c, (int64_t)r + c.offset);
        bool mn = A.op == OP_ARGMIN_R64;
        atomic_arg_r64((unsigned long long*)d, c, ord64(c, e, mn), (uint32_t)r, mn);
      }
      break;
    }
    default: break;
  }
}

}  // namespace gb
