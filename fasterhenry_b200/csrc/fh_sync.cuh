// Bounded inter-CTA barrier for cooperative launches whose CTAs form
// independent groups (one group per matrix or per matrix and right-hand
// side).  Only the CTAs of one group meet; each group has its own counter.
#pragma once

#include <cuda_runtime.h>

namespace fhb {

// Unsigned words per group barrier: one 128-byte line each.
constexpr int kGroupBarrierStride = 32;
constexpr long long kGroupBarrierSpin = 1LL << 22;

// Sense-reversing barrier of the `expected` CTAs that share `bar` (bar[0]
// counts arrivals, bar[1] is the generation).  Every thread of the CTA must
// call it.  A wait that runs past its iteration limit, or that sees the error
// flag raised by another CTA, sets the flag and returns false; the caller
// then returns without touching shared data again.
__device__ __forceinline__ bool group_barrier(unsigned *bar, unsigned expected, int *error) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *vgen = bar + 1;
        const unsigned gen = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(bar, 1u);
        int ok = 1;
        if (arrived == expected - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long i = 0;
            while (*vgen == gen) {
                if (++i > kGroupBarrierSpin || *(volatile int *)error) {
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        if (!ok) atomicExch(error, 1);
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

}  // namespace fhb
