// Launchers of the scan / radix sort / cell-offset kernels (sort.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace gpgmp {

// scratch of one exclusive scan of n values: a tile counter, an error word and one
// status word per kScanTile (16384) values; the error word sits at byte scan_error_flag_offset()
size_t scan_scratch_bytes(int64_t n);
int scan_error_flag_offset();
cudaError_t scan_exclusive_u32(const uint32_t* in, uint32_t* out, int64_t n, void* scratch, cudaStream_t st);

struct SortLayout {
    int digit_bits;   // 8, or 10 where that saves a pass; hist is [passes][1 << digit_bits]
    int passes;
    int64_t tiles;
    size_t off_hist, off_counters, off_look, off_alt_keys, off_alt_vals, bytes;
};
// scratch layout of one radix sort; the error word is the uint32 at off_counters + 16
SortLayout sort_layout(int64_t n, int key_bits);
// With cell_count (zeroed by the caller), the last pass also adds the number of keys
// equal to each c < ncells into cell_count[c].
cudaError_t radix_sort_pairs_u32(const uint32_t* kin, const uint32_t* vin, uint32_t* kout, uint32_t* vout, int64_t n,
                                 int key_bits, void* scratch, cudaStream_t st, uint32_t* cell_count = nullptr,
                                 int64_t ncells = 0);
// The same in two halves around a caller's kernel that adds the digit counts of every
// pass ([passes][1 << digit_bits], radix_sort_hist) while it writes the keys: begin clears the
// scratch, finish sorts.  With cell_count (zeroed by the caller), the last pass also
// adds the number of keys equal to each c < ncells into cell_count[c].
cudaError_t radix_sort_begin(int64_t n, int key_bits, void* scratch, cudaStream_t st);
uint32_t* radix_sort_hist(int64_t n, int key_bits, void* scratch);
cudaError_t radix_sort_finish(const uint32_t* kin, const uint32_t* vin, uint32_t* kout, uint32_t* vout, int64_t n,
                              int key_bits, void* scratch, cudaStream_t st, uint32_t* cell_count = nullptr,
                              int64_t ncells = 0);

// count[c] = number of keys equal to c (keys at or past ncells are not counted)
cudaError_t cell_counts_u32(const uint32_t* sorted_keys, int64_t n, int64_t ncells, uint32_t* count, cudaStream_t st);
// count as above, start = exclusive scan of count
cudaError_t cell_offsets_u32(const uint32_t* sorted_keys, int64_t n, int64_t ncells, uint32_t* start, uint32_t* count,
                             void* scan_scratch, cudaStream_t st);
// the reference's [left, right] cell indices from start and count
cudaError_t left_right_u32(const uint32_t* start, const uint32_t* count, int64_t ncells, uint32_t* left,
                           uint32_t* right, cudaStream_t st);

// gpgmp_population_maintain with the number of individuals created (births_out,
// may be NULL): they took the first births_out ids of the old pool (population.cu)
int population_maintain(const uint32_t* keys, const uint32_t* ids, int64_t n_active, const uint32_t* cell_start,
                        const uint32_t* cell_count, const int32_t* goal, int64_t ncells, const uint32_t* pool,
                        int64_t n_pool, uint32_t seed, uint32_t step, uint32_t* keys_out, uint32_t* ids_out,
                        int64_t capacity_out, uint32_t* pool_out, int64_t pool_capacity, uint32_t* start_out,
                        int64_t* n_active_out, int64_t* n_pool_out, int64_t* births_out, void* scratch,
                        size_t scratch_bytes, void* stream);

}  // namespace gpgmp
