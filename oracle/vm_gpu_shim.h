/*
 * ORACLE / TEST INFRASTRUCTURE ONLY (force-included when oracle/Makefile
 * compiles the reference's src/vm/vm_gpu.cu into _ref/libvirg_refgpu.so).
 *
 * The reference passes its __constant__ symbols as `(char*)&symbol` to
 * cudaMemcpyToSymbol / cudaMemcpyToSymbolAsync / cudaMemcpyFromSymbol
 * (src/vm/vm_gpu.cu:121-129 and later), the form of the runtime API before
 * CUDA 5, where a char pointer named the symbol.  With CUDA 12 that argument
 * selects the C++ template overloads, which take the address of the pointer
 * itself and fail with "invalid device symbol".  These wrappers hand the
 * symbol's address to the C entry points instead, so the reference code runs
 * unmodified.
 */
#ifndef VGREF_SHIM_H
#define VGREF_SHIM_H
#include <cuda_runtime_api.h>

static inline cudaError_t vgref_to_symbol(const char *sym, const void *src, size_t n, size_t off,
	enum cudaMemcpyKind kind)
{
	return cudaMemcpyToSymbol((const void *)sym, src, n, off, kind);
}
static inline cudaError_t vgref_to_symbol_async(const char *sym, const void *src, size_t n, size_t off,
	enum cudaMemcpyKind kind, cudaStream_t st)
{
	return cudaMemcpyToSymbolAsync((const void *)sym, src, n, off, kind, st);
}
static inline cudaError_t vgref_from_symbol(void *dst, const char *sym, size_t n, size_t off,
	enum cudaMemcpyKind kind)
{
	return cudaMemcpyFromSymbol(dst, (const void *)sym, n, off, kind);
}
#define cudaMemcpyToSymbol vgref_to_symbol
#define cudaMemcpyToSymbolAsync vgref_to_symbol_async
#define cudaMemcpyFromSymbol vgref_from_symbol
#endif
