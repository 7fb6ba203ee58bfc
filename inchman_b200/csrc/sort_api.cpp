// C ABI of the scan / sort / cell-offset primitives (sort.cu).  Device pointers;
// the caller passes the scratch buffer (size from the *_scratch_bytes queries).
#include <cuda_runtime.h>
#include "sort_kernels.h"
#include "host_common.h"
#include "../../include/gpgmp_c.h"

using namespace gpgmp;

#define CK(expr)                                                                                              \
    do {                                                                                                      \
        cudaError_t e_ = (expr);                                                                              \
        if (e_ != cudaSuccess) return set_error(GPGMP_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_));    \
    } while (0)

extern "C" {

int gpgmp_scan_scratch_bytes(int64_t n, size_t* bytes) {
    if (!bytes || n < 0) return set_error(GPGMP_ERR_INVALID, "bad argument");
    *bytes = scan_scratch_bytes(n);
    return GPGMP_OK;
}

int gpgmp_exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, void* scratch, size_t scratch_bytes,
                             void* stream) {
    if (n < 0 || (n > 0 && (!in || !out || !scratch))) return set_error(GPGMP_ERR_INVALID, "bad argument");
    if (n > ((int64_t)1 << 34)) return set_error(GPGMP_ERR_INVALID, "n too large");
    if (scratch_bytes < scan_scratch_bytes(n)) return set_error(GPGMP_ERR_INVALID, "scratch too small");
    CK(scan_exclusive_u32(in, out, n, scratch, (cudaStream_t)stream));
    return GPGMP_OK;
}

int gpgmp_sort_scratch_bytes(int64_t n, int32_t key_bits, size_t* bytes) {
    if (!bytes || n < 0 || key_bits < 1 || key_bits > 32) return set_error(GPGMP_ERR_INVALID, "bad argument");
    *bytes = sort_layout(n, key_bits).bytes;
    return GPGMP_OK;
}

int gpgmp_sort_pairs_u32(const uint32_t* kin, const uint32_t* vin, uint32_t* kout, uint32_t* vout, int64_t n,
                         int32_t key_bits, void* scratch, size_t scratch_bytes, void* stream) {
    if (n < 0 || key_bits < 1 || key_bits > 32) return set_error(GPGMP_ERR_INVALID, "bad argument");
    if (n > ((int64_t)1 << 30) - 1) return set_error(GPGMP_ERR_INVALID, "n above 2^30 - 1");
    if (n > 0 && (!kin || !vin || !kout || !vout || !scratch)) return set_error(GPGMP_ERR_INVALID, "NULL pointer");
    if (scratch_bytes < sort_layout(n, key_bits).bytes) return set_error(GPGMP_ERR_INVALID, "scratch too small");
    CK(radix_sort_pairs_u32(kin, vin, kout, vout, n, key_bits, scratch, (cudaStream_t)stream));
    return GPGMP_OK;
}

int gpgmp_cell_offsets(const uint32_t* sorted_keys, int64_t n, int64_t ncells, uint32_t* start, uint32_t* count,
                       void* scratch, size_t scratch_bytes, void* stream) {
    if (n < 0 || ncells <= 0 || !start || !count || !scratch) return set_error(GPGMP_ERR_INVALID, "bad argument");
    if (n > 0 && !sorted_keys) return set_error(GPGMP_ERR_INVALID, "NULL keys");
    if (scratch_bytes < scan_scratch_bytes(ncells)) return set_error(GPGMP_ERR_INVALID, "scratch too small");
    CK(cell_offsets_u32(sorted_keys, n, ncells, start, count, scratch, (cudaStream_t)stream));
    return GPGMP_OK;
}

int gpgmp_cell_indices(const uint32_t* start, const uint32_t* count, int64_t ncells, uint32_t* left, uint32_t* right,
                       void* stream) {
    if (ncells <= 0 || !start || !count || !left || !right) return set_error(GPGMP_ERR_INVALID, "bad argument");
    CK(left_right_u32(start, count, ncells, left, right, (cudaStream_t)stream));
    return GPGMP_OK;
}

int gpgmp_scratch_status(const void* scratch, int32_t kind, int64_t n, int32_t key_bits, int32_t* status) {
    if (!scratch || !status) return set_error(GPGMP_ERR_INVALID, "bad argument");
    size_t off = kind == 0 ? (size_t)scan_error_flag_offset() : sort_layout(n, key_bits).off_counters + 16;
    int v = 0;
    CK(cudaMemcpy(&v, (const char*)scratch + off, sizeof(int), cudaMemcpyDeviceToHost));
    *status = v ? GPGMP_ERR_TIMEOUT : GPGMP_OK;
    return GPGMP_OK;
}

}  // extern "C"
