/* gsrb/cudaLocks.h -- drop-in host API of the Heterosync cudaLocks layer.
 *
 * Same names, argument meanings and return values as the reference
 * (Heterosync/cudaLocks.h:4-27, cudaLocks.cu:3-102, cudaLocksMutex*.cu:4-11,
 * cudaLocksSemaphoreSpin.cu:6-29, cudaLocksSemaphoreEBO.cu:4-28), exported by
 * libgsrb.so with C linkage:
 *   - cudaLocksInit returns cudaErrorInitializationError for non-positive
 *     arguments (cudaLocks.cu:13-15), cudaSuccess otherwise; allocation failures
 *     are returned instead of exiting;
 *   - cpuLockData is pinned host memory that kernels read through unified
 *     addressing, as in the reference (cudaLocks.cu:11);
 *   - buffer sizes follow the reference (arrayStride = (maxBlocks + NUM_SM) / 16 * 16);
 *     the mutex ring buffers start as 1, -1, -1, ... per stride (cudaLocks.cu:50-63).
 * Difference: every buffer carries a 128-byte header whose first word is a status
 * word written by the bounded waits of the device functions
 * (gsrb/cudaLocks.cuh); gsrb_cudalocks_status() reads and clears them.
 */
#ifndef GSRB_CUDALOCKS_H_
#define GSRB_CUDALOCKS_H_
#include <cuda_runtime_api.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

typedef struct cudaLockData {
  int maxBufferSize;
  int arrayStride;
  int mutexCount;
  int semaphoreCount;
  unsigned int* barrierBuffers;
  int* mutexBuffers;
  unsigned int* mutexBufferHeads;
  unsigned int* mutexBufferTails;
  unsigned int* semaphoreBuffers;
} cudaLockData_t;

typedef unsigned int cudaMutex_t;
typedef unsigned int cudaSemaphore_t;

#ifdef __cplusplus
extern "C" {
#endif

/* The single lock-state instance (Heterosync/cudaLocks.h:22). */
extern cudaLockData_t* cpuLockData;

cudaError_t cudaLocksInit(const int maxBlocksPerKernel, const int numMutexes, const int numSemaphores,
                          const bool pageAlign, const int NUM_SM);
cudaError_t cudaLocksDestroy(void);

cudaError_t cudaMutexCreateSpin(cudaMutex_t* const handle, const int mutexNumber);
cudaError_t cudaMutexCreateEBO(cudaMutex_t* const handle, const int mutexNumber);
cudaError_t cudaMutexCreateFA(cudaMutex_t* const handle, const int mutexNumber);
cudaError_t cudaMutexCreateSleep(cudaMutex_t* const handle, const int mutexNumber);
cudaError_t cudaSemaphoreCreateSpin(cudaSemaphore_t* const handle, const int semaphoreNumber,
                                    const unsigned int count, const int NUM_SM);
cudaError_t cudaSemaphoreCreateEBO(cudaSemaphore_t* const handle, const int semaphoreNumber,
                                   const unsigned int count, const int NUM_SM);

/* Synchronous: first device status code recorded in any lock buffer (0 = none), then cleared. */
unsigned int gsrb_cudalocks_status(void);

#ifdef __cplusplus
}
#endif
#endif
