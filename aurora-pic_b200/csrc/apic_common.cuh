// Shared host/device helpers of the aurora-pic B200 library.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "aurorapic_b200.h"

namespace apic {

// A failure that maps onto an apic_status at the C ABI.
struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& what) : std::runtime_error(what), status(s) {}
};

inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw Error(APIC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define APIC_CUDA(call) ::apic::cuda_check((call), #call)

inline void require(bool ok, const std::string& what, int status = APIC_ERR_INVALID) {
    if (!ok) throw Error(status, what);
}

// Fixed-point charge accumulation: contributions are rounded once to
// multiples of 2^-scale_bits and summed in 64-bit integers, so the deposited
// density does not depend on the order in which particles are processed.
__device__ __forceinline__ long long to_fixed(double value, double scale) {
    return __double2ll_rn(value * scale);
}

// Waits on the handle's stream without blocking forever: polls the event
// until it completes or `seconds` elapse.
cudaError_t bounded_wait(cudaStream_t stream, double seconds);

// Device error word -> apic_status (first matching bit wins).
int status_from_device(unsigned word);
std::string describe_device_error(unsigned word);

}  // namespace apic
