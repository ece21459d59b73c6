/*
 * ORACLE / TEST INFRASTRUCTURE ONLY (linked into oracle/_ref/libvirg_host.so).
 *
 * virg_init (src/init.c:45) calls
 *   cudaSetDeviceFlags(cudaDeviceMapHost | cudaDeviceScheduleSpin |
 *                      cudaDeviceScheduleBlockingSync)
 * and CUDA 12.9 rejects the two scheduling policies together as an invalid
 * argument, so the reference host library cannot initialise against the real
 * runtime.  This wrapper keeps MapHost and one scheduling policy
 * (BlockingSync) and forwards to the CUDA runtime, so the rest of virg_init
 * runs unmodified.
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <cuda_runtime_api.h>

cudaError_t cudaSetDeviceFlags(unsigned int flags)
{
	static cudaError_t (*real)(unsigned int) = 0;
	if (!real)
		real = (cudaError_t (*)(unsigned int))dlsym(RTLD_NEXT, "cudaSetDeviceFlags");
	if (!real)
		return cudaErrorUnknown;
	unsigned sched = flags & cudaDeviceScheduleMask;
	if (sched & cudaDeviceScheduleBlockingSync)
		sched = cudaDeviceScheduleBlockingSync;
	return real((flags & ~cudaDeviceScheduleMask) | sched);
}
