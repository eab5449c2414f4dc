// gsrb/compat.h -- reference-named host entry points (C++ linkage, like the
// reference headers) so that the reference's own drivers link against libgsrb
// unchanged:
//   int  reduce(const int* arr, unsigned N, unsigned threads_per_block)
//        Reduce/reduce.cuh:19 -- host array in, int sum out, prints
//        "time (ms) is %f" like Reduce/reduce_gsrb.cu:396
//   void sum_scan_blelloch(unsigned* d_out, unsigned* d_in, size_t numElems)
//        scan/scan.h:16-18 -- device pointers, exclusive uint32 scan, prints
//        "Kernel time (ms) %f" like scan/scan_gsrb.cu:785
//   void sum_scan_naive(unsigned* d_out, const unsigned* d_in, size_t numElems)
//        scan/scan.h:12-14
// They run on a process-wide default context (device 0 or the current device)
// and, unlike the reference, work for any N (the grid is fixed and always
// co-resident) and never exit the process on error (errors are printed).
#pragma once
#include <stddef.h>

int reduce(const int* arr, unsigned int N, unsigned int threads_per_block);
void sum_scan_blelloch(unsigned int* d_out, unsigned int* d_in, const size_t numElems);
void sum_scan_naive(unsigned int* const d_out, const unsigned int* const d_in, const size_t numElems);
