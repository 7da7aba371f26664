// Test-only: host stand-ins for the CUDA qualifiers and builtins that
// hera_b200/csrc/hera_device.cuh names, so that its gap DP (sw_align_bits,
// sw_align_reg) compiles for the host in the CPU suite.  Only the
// single-thread integer functions are meaningful here: the warp-level
// builtins (shuffles, ballots, byte permutes) are placeholders that let the
// rest of the header compile; nothing the checks call uses them.
#pragma once
#include <cstdint>
#include <cstring>
#define __device__
#define __host__
#define __forceinline__ inline
#define __global__
#define __restrict__
struct uint2 {
	uint32_t x, y;
};
struct uint4 {
	uint32_t x, y, z, w;
};
struct int2 {
	int x, y;
};
static inline uint2 make_uint2(uint32_t a, uint32_t b) { return uint2{a, b}; }
static inline uint4 make_uint4(uint32_t a, uint32_t b, uint32_t c, uint32_t d) { return uint4{a, b, c, d}; }
static inline int2 make_int2(int a, int b) { return int2{a, b}; }
template <class T>
static inline T __ldg(const T *p)
{
	return *p;
}
static inline int __ffs(uint32_t x) { return x ? __builtin_ctz(x) + 1 : 0; }
static inline int __clz(uint32_t x) { return x ? __builtin_clz(x) : 32; }
static inline unsigned __byte_perm(unsigned, unsigned, unsigned) { return 0; }
static inline unsigned __ballot_sync(unsigned, int) { return 0; }
static inline int __reduce_max_sync(unsigned, int v) { return v; }
static inline int __reduce_min_sync(unsigned, int v) { return v; }
template <class T>
static inline T __shfl_sync(unsigned, T v, int)
{
	return v;
}
template <class T>
static inline T __shfl_up_sync(unsigned, T v, int)
{
	return v;
}
static inline void __syncwarp(unsigned = 0xffffffffu) {}
static inline int __viaddmin_s32(int a, int b, int c) { return a + b < c ? a + b : c; }
static inline int __vimax3_s32_relu(int a, int b, int c)
{
	int m = a > b ? a : b;
	m = m > c ? m : c;
	return m > 0 ? m : 0;
}
static inline int max(int a, int b) { return a > b ? a : b; }
static inline int min(int a, int b) { return a < b ? a : b; }
struct HostDim3 {
	unsigned x, y, z;
};
static HostDim3 threadIdx{0, 0, 0};
