// Radix sorts, scans and reductions over device arrays (CUB library calls, stream-ordered
// on the solver's stream, scratch kept in the solver).
#include <cub/cub.cuh>

#include "fmm_solver.cuh"

namespace fmmb200 {

void sort_pairs_u64(SolverBase& s, const unsigned long long* kin, unsigned long long* kout,
                    const int* vin, int* vout, int n, int end_bit, int begin_bit) {
  if (n <= 0) return;
  size_t bytes = 0;
  FMM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, n, begin_bit,
                                           end_bit, s.stream));
  s.cub_tmp.ensure(bytes);
  FMM_CUDA(cub::DeviceRadixSort::SortPairs(s.cub_tmp.p, bytes, kin, kout, vin, vout, n,
                                           begin_bit, end_bit, s.stream));
}

void sort_keys_u64(SolverBase& s, const unsigned long long* kin, unsigned long long* kout,
                   int n, int end_bit) {
  if (n <= 0) return;
  size_t bytes = 0;
  FMM_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, bytes, kin, kout, n, 0, end_bit, s.stream));
  s.cub_tmp.ensure(bytes);
  FMM_CUDA(cub::DeviceRadixSort::SortKeys(s.cub_tmp.p, bytes, kin, kout, n, 0, end_bit,
                                          s.stream));
}

void segmented_sort_pairs_u64(SolverBase& s, const unsigned long long* kin,
                              unsigned long long* kout, const int* vin, int* vout, int n,
                              int nseg, const int* begin, const int* end, int end_bit) {
  if (n <= 0) return;
  size_t bytes = 0;
  FMM_CUDA(cub::DeviceSegmentedRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, n, nseg,
                                                    begin, end, 0, end_bit, s.stream));
  s.cub_tmp.ensure(bytes);
  FMM_CUDA(cub::DeviceSegmentedRadixSort::SortPairs(s.cub_tmp.p, bytes, kin, kout, vin, vout, n,
                                                    nseg, begin, end, 0, end_bit, s.stream));
}

void sort_pairs_u32(SolverBase& s, const unsigned* kin, unsigned* kout, const int* vin,
                    int* vout, int n, int end_bit, DevArr<char>* tmp) {
  if (n <= 0) return;
  DevArr<char>& t = tmp ? *tmp : s.cub_tmp;
  size_t bytes = 0;
  FMM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, n, 0, end_bit,
                                           s.stream));
  t.ensure(bytes);
  FMM_CUDA(cub::DeviceRadixSort::SortPairs(t.p, bytes, kin, kout, vin, vout, n, 0, end_bit,
                                           s.stream));
}

void exclusive_sum_int(SolverBase& s, const int* in, int* out, int n, DevArr<char>* tmp) {
  if (n <= 0) return;
  DevArr<char>& t = tmp ? *tmp : s.cub_tmp;
  size_t bytes = 0;
  FMM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, s.stream));
  t.ensure(bytes);
  FMM_CUDA(cub::DeviceScan::ExclusiveSum(t.p, bytes, in, out, n, s.stream));
}

void sum_u64(SolverBase& s, const unsigned long long* in, unsigned long long* out, int n) {
  size_t bytes = 0;
  FMM_CUDA(cub::DeviceReduce::Sum(nullptr, bytes, in, out, n, s.stream));
  s.cub_tmp.ensure(bytes);
  FMM_CUDA(cub::DeviceReduce::Sum(s.cub_tmp.p, bytes, in, out, n, s.stream));
}

}  // namespace fmmb200
