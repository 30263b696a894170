// qssb_internal.h - host-side helpers shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../../include/qssb.h"
#include "qssb_device.cuh"

namespace qssb {

// Records a thread-local error message and returns `code`.
int set_error(int code, const char* msg);
int set_cuda_error(cudaError_t err, const char* where);
// Multiprocessor count of the current device (cached per device).
int device_sm_count();
// Probe constants of one candidate (host side; cos/sin of 2 phi12 in FP64).
Probe make_probe(const qssb_calibration_t& cal, const qssb_aberrations_t& ab);
// Validates a calibration; returns QSSB_OK or an error code (message set).
int validate_calibration(const qssb_calibration_t* cal, const char* who);
// Tile-shape variant carried in flags (QSSB_FLAG_VARIANT); 0 = built-in shape.
inline int flag_variant(int32_t flags) {
    return (int)((flags >> QSSB_FLAG_VARIANT_SHIFT) & QSSB_FLAG_VARIANT_MAX);
}

// Requested chunk count carried in flags (QSSB_FLAG_CHUNKS); 0 = built-in plan.
inline int flag_chunks(int32_t flags) {
    return (int)((flags >> QSSB_FLAG_CHUNKS_SHIFT) & QSSB_FLAG_CHUNKS_MAX);
}

// Counts one kernel launch made by this library (every <<< >>> site calls it
// right after the launch): qssb_kernel_launches reports the running total.
void note_launch();

}  // namespace qssb

#define QSSB_STR2(x) #x
#define QSSB_STR(x) QSSB_STR2(x)
#define CUDA_TRY(expr)                                                          \
    do {                                                                        \
        cudaError_t _e = (expr);                                                \
        if (_e != cudaSuccess)                                                  \
            return ::qssb::set_cuda_error(_e, __FILE__ ":" QSSB_STR(__LINE__)); \
    } while (0)
