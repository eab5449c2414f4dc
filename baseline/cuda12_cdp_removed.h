/* Force-included when the reference's Lonestar kernel files are compiled for
 * sm_100a (the reference's own GPU programs, the timing baseline and the source of
 * golden outputs).  Each of those files keeps a
 * dead kernel, gg_main_pipe_1_gpu, whose launch is commented out and which
 * calls cudaDeviceSynchronize() from device code -- dynamic-parallelism
 * synchronisation that CUDA 12 removed.  In the device pass the name is mapped
 * to a function that returns cudaErrorNotSupported, so the dead kernel
 * compiles; host code keeps the real cudaDeviceSynchronize. */
#pragma once
#if defined(__CUDA_ARCH__)
static __host__ __device__ __forceinline__ cudaError_t gsrb_removed_device_sync(void) {
  return cudaErrorNotSupported;
}
#define cudaDeviceSynchronize gsrb_removed_device_sync
#endif
