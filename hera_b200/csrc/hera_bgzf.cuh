// hera_bgzf.cuh -- BGZF compression of a byte stream on the device (the BAM
// container hera's bam_write produces on the host, src/hash_align.c:48-136):
// one thread per 64 KiB block runs hera_bgzf_core.h's encoder with its hash
// table and the CRC table in shared memory; a scan of the block sizes and a
// gather pack the blocks back to back.
#include "hera_bgzf_core.h"

namespace bgzfk {

constexpr int TPB = 8;                      // blocks (threads) per CTA
constexpr int HB = 12;                      // 4096-entry tables: 8 KiB a thread
constexpr size_t SMEM = 1024 + (size_t)TPB * (sizeof(uint16_t) << HB);

__global__ void __launch_bounds__(TPB) k_bgzf(const uint8_t *__restrict__ in, int64_t n, int64_t nb,
					       uint8_t *__restrict__ slots, unsigned long long *__restrict__ size)
{
	extern __shared__ __align__(16) uint8_t sm[];
	uint32_t *crc_t = reinterpret_cast<uint32_t *>(sm);
	if (threadIdx.x == 0)
		bgzf::crc_table(crc_t);
	__syncthreads();
	const int64_t k = (int64_t)blockIdx.x * TPB + threadIdx.x;
	if (k > nb)
		return;
	if (k == nb) {
		size[nb] = 0;
		return;
	}
	uint16_t *table = reinterpret_cast<uint16_t *>(sm + 1024) + (size_t)threadIdx.x * (1u << HB);
	const int64_t a = k * bgzf::BLOCK_IN;
	const int len = (int)(n - a < bgzf::BLOCK_IN ? n - a : bgzf::BLOCK_IN);
	size[k] = (unsigned long long)bgzf::block<HB>(in + a, len, slots + (size_t)k * bgzf::BLOCK_MAX, table, crc_t);
}

// block k's bytes to out + off[k] (a warp a block, 16-byte words where aligned)
__global__ void k_bgzf_gather(const uint8_t *__restrict__ slots, const unsigned long long *__restrict__ off,
			      int64_t nb, uint8_t *__restrict__ out)
{
	const int64_t k = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
	if (k >= nb)
		return;
	const int lane = threadIdx.x & 31;
	const uint8_t *s = slots + (size_t)k * bgzf::BLOCK_MAX;
	uint8_t *d = out + off[k];
	const int len = (int)(off[k + 1] - off[k]);
	for (int i = lane; i < len; i += 32)
		d[i] = s[i];
}

}  // namespace bgzfk

// compress d_in[0 .. n) (device) into d_out (device, cap bytes) on `st`;
// *used = the BGZF bytes.  Scratch: (blocks) x 64 KiB slots and sizes.
static int bgzf_run(hera_gpu_ctx *ctx, const uint8_t *d_in, uint64_t n, uint8_t *d_out, uint64_t cap,
		    uint64_t *used, cudaStream_t st, float *kernel_ms)
{
	const int64_t nb = (int64_t)((n + bgzf::BLOCK_IN - 1) / bgzf::BLOCK_IN);
	*used = 0;
	if (nb == 0)
		return HERA_GPU_OK;
	uint8_t *slots = nullptr;
	unsigned long long *size = nullptr, *off = nullptr;
	void *tmp = nullptr;
	size_t tmp_bytes = 0;
	cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, (unsigned long long *)nullptr, (unsigned long long *)nullptr,
				      nb + 1, st);
	cudaError_t e;
	auto release = [&] { cudaFree(slots); cudaFree(size); cudaFree(off); cudaFree(tmp); };
	if ((e = cudaMalloc(&slots, (size_t)nb * bgzf::BLOCK_MAX)) != cudaSuccess ||
	    (e = cudaMalloc(&size, (nb + 1) * 8ull)) != cudaSuccess || (e = cudaMalloc(&off, (nb + 1) * 8ull)) != cudaSuccess ||
	    (e = cudaMalloc(&tmp, tmp_bytes + 16)) != cudaSuccess) {
		release();
		return fail(ctx, HERA_GPU_ENOMEM, "BGZF scratch", e);
	}
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	cudaEventRecord(e0, st);
	bgzfk::k_bgzf<<<(unsigned)((nb + 1 + bgzfk::TPB - 1) / bgzfk::TPB), bgzfk::TPB, bgzfk::SMEM, st>>>(
		d_in, (int64_t)n, nb, slots, size);
	cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, size, off, nb + 1, st);
	unsigned long long total = 0;
	if ((e = cudaMemcpyAsync(&total, off + nb, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
	    (e = cudaStreamSynchronize(st)) != cudaSuccess) {
		release();
		cudaEventDestroy(e0);
		cudaEventDestroy(e1);
		return fail(ctx, HERA_GPU_ECUDA, "BGZF blocks", e);
	}
	*used = total;
	int rc = HERA_GPU_OK;
	if (total > cap) {
		rc = fail(ctx, HERA_GPU_ECAPACITY, "BGZF output buffer too small (*out_len holds the size)");
	} else {
		bgzfk::k_bgzf_gather<<<blocks_for(nb * 32, 256), 256, 0, st>>>(slots, off, nb, d_out);
		cudaEventRecord(e1, st);
		if ((e = cudaStreamSynchronize(st)) != cudaSuccess)
			rc = fail(ctx, HERA_GPU_ECUDA, "BGZF gather", e);
		else if (kernel_ms)
			cudaEventElapsedTime(kernel_ms, e0, e1);
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	release();
	return rc;
}

extern "C" int hera_gpu_bgzf(hera_gpu_ctx *ctx, const uint8_t *in, uint64_t n, uint8_t *out, uint64_t cap,
			     uint64_t *out_len, float *kernel_ms)
{
	if (!ctx || (n && (!in || !out)) || !out_len)
		return fail(ctx, HERA_GPU_EINVAL, "bad argument");
	*out_len = 0;
	if (n == 0)
		return HERA_GPU_OK;
	if (cudaSetDevice(ctx->device) != cudaSuccess)
		return fail(ctx, HERA_GPU_ENODEV, "cudaSetDevice");
	static bool attr_set = false;
	if (!attr_set) {
		if (cudaFuncSetAttribute(bgzfk::k_bgzf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bgzfk::SMEM) !=
		    cudaSuccess)
			return fail(ctx, HERA_GPU_ECUDA, "BGZF kernel shared-memory size");
		attr_set = true;
	}
	const uint64_t nb = (n + bgzf::BLOCK_IN - 1) / bgzf::BLOCK_IN;
	const uint64_t worst = nb * bgzf::BLOCK_MAX;
	uint8_t *d_in = nullptr, *d_out = nullptr;
	cudaError_t e;
	if ((e = cudaMalloc(&d_in, n)) != cudaSuccess || (e = cudaMalloc(&d_out, worst)) != cudaSuccess) {
		cudaFree(d_in);
		return fail(ctx, HERA_GPU_ENOMEM, "BGZF buffers", e);
	}
	const cudaStream_t st = ctx->stream;
	int rc = HERA_GPU_OK;
	uint64_t used = 0;
	if ((e = cudaMemcpyAsync(d_in, in, n, cudaMemcpyHostToDevice, st)) != cudaSuccess)
		rc = fail(ctx, HERA_GPU_ECUDA, "BGZF input copy", e);
	if (rc == HERA_GPU_OK)
		rc = bgzf_run(ctx, d_in, n, d_out, worst, &used, st, kernel_ms);
	*out_len = used;
	if (rc == HERA_GPU_OK && used > cap)
		rc = fail(ctx, HERA_GPU_ECAPACITY, "BGZF output buffer too small (*out_len holds the size)");
	if (rc == HERA_GPU_OK &&
	    ((e = cudaMemcpyAsync(out, d_out, used, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
	     (e = cudaStreamSynchronize(st)) != cudaSuccess))
		rc = fail(ctx, HERA_GPU_ECUDA, "BGZF output copy", e);
	cudaFree(d_in);
	cudaFree(d_out);
	return rc;
}
