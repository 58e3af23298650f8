// ref_driver.cu -- C entry points around the reference's compiled search.
//
// TEST INFRASTRUCTURE ONLY.  build_ref.sh compiles this file together with the
// reference's unmodified emitter/src/native/backtracking/sorting_search.cu and
// slot_manager.cu into oracle/_ref/libtd16ref.so.  Tests load it to produce
// verdict and witness fixtures from the reference kernel itself.
#include <cstdint>
#include <cstdio>
#include <exception>
#include <string>
#include <vector>

#include "backtracking/slot_manager.cuh"
#include "backtracking/sorting_search.cuh"
#include "core/cuda_error.cuh"

static void put(char *err, size_t len, const char *msg) {
    if (err && len) std::snprintf(err, len, "%s", msg);
}

extern "C" int ref_init(int slots, int device, unsigned long long budget, char *err, size_t errlen) {
    try {
        initGpuSortSlots(slots, std::vector<int>{device}, (size_t)budget);
        return 0;
    } catch (const std::exception &e) {
        put(err, errlen, e.what());
        return 1;
    }
}

// Mirrors jni_sorter.cu:49-117 (minRate travels as float, widened to double).
extern "C" int ref_search(const uint8_t *beta, const uint8_t *omega, int n, int init, float min_rate,
                          int max_moves, int full, int slot, int max_warps, int16_t *out_ijk,
                          int *out_depth, char *err, size_t errlen) {
    try {
        clearCudaRuntimePoisoned();
        std::vector<short> b(n), o(n);
        for (int i = 0; i < n; ++i) {
            b[i] = (short)(beta[i] & 0xFF);
            o[i] = (short)(omega[i] & 0xFF);
        }
        if (getGpuSortSlotDevice(slot) < 0) throw std::invalid_argument("invalid GPU sorting slot");
        cudaStream_t stream = getGpuSortSlotStream(slot);
        const auto moves = performGpuSortingSearch(b, o, init, (double)min_rate, max_moves, full != 0,
                                                   stream, slot, max_warps);
        for (size_t d = 0; d < moves.size(); ++d) {
            out_ijk[3 * d] = moves[d].firstIndex;
            out_ijk[3 * d + 1] = moves[d].secondIndex;
            out_ijk[3 * d + 2] = moves[d].thirdIndex;
        }
        *out_depth = (int)moves.size();
        return 0;
    } catch (const std::exception &e) {
        put(err, errlen, e.what());
        *out_depth = 0;
        return 2;
    }
}

extern "C" int ref_destroy() {
    try {
        destroyGpuSortSlots();
        return 0;
    } catch (...) {
        return 1;
    }
}
