/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.  Nothing in the product links this file.
 *
 * Host-only stand-ins for the eight CUDA runtime calls that the reference's
 * non-GPU sources make (src/init.c:45-80, src/close.c:20-40 and the
 * VIRG_CUDCHK macro, src/virginian.h:130-149), so the reference's CPU virtual
 * machines run on a machine without a GPU.  Pinned/mapped host allocations
 * become plain malloc; device allocations become malloc as well (the CPU VMs
 * never touch them).  The symbols are hidden by oracle/ref.map so they never
 * interpose on a real libcudart loaded in the same process.
 *
 * Also provides stubs for virg_vm_gpu/virg_gpu_getsizes (src/virginian.h:620-622)
 * because src/vm/execute.c:86 references the GPU VM; the oracle library never
 * takes that branch (use_gpu stays 0) and fails loudly if it does.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <cuda_runtime_api.h>

#include "virginian.h"

cudaError_t cudaSetDeviceFlags(unsigned int flags) { (void)flags; return cudaSuccess; }
cudaError_t cudaSetDevice(int device) { (void)device; return cudaSuccess; }
cudaError_t cudaGetLastError(void) { return cudaSuccess; }
const char *cudaGetErrorString(cudaError_t e) { (void)e; return "oracle cuda stub"; }
cudaError_t cudaHostAlloc(void **p, size_t size, unsigned int flags)
{
	(void)flags;
	*p = malloc(size);
	return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaFreeHost(void *p) { free(p); return cudaSuccess; }
cudaError_t cudaMalloc(void **p, size_t size)
{
	/* the reference reserves VIRG_GPU_TABLETS device slots (src/init.c:72-80);
	 * the CPU VMs never read them, so hand back a small host block */
	(void)size;
	*p = malloc(64);
	return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaFree(void *p) { free(p); return cudaSuccess; }
cudaError_t cudaMemset(void *p, int v, size_t n) { (void)p; (void)v; (void)n; return cudaSuccess; }
cudaError_t cudaThreadExit(void) { return cudaSuccess; }

int virg_vm_gpu(virginian *v, virg_vm *vm, virg_tablet_meta **tab,
	virg_tablet_meta **res, unsigned num_tablets)
{
	(void)v; (void)vm; (void)tab; (void)res; (void)num_tablets;
	fprintf(stderr, "oracle library: the GPU VM is not part of the oracle\n");
	abort();
}

const size_t *virg_gpu_getsizes(void)
{
	return &virg_testsizes[0];
}
