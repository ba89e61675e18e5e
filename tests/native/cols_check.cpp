// cols_check.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Reads a batch_*/bits directory with the library's column reader
// (kgio::load_matrix_packed, supergwas_b200/csrc/kgwas_io.cpp) into packed
// k-mer-major rows, so that the CPU test suite can compare them with the
// packing of the rows the columns were written from.
#include <string>
#include <vector>

#include "../../supergwas_b200/csrc/kgwas_io.hpp"

extern "C" void cols_read(const char* bits_dir, const int* idxs, int n, unsigned long N, int threads,
                          uint64_t* out) {
  std::vector<int> ix(idxs, idxs + n);
  kgio::load_matrix_packed(bits_dir, ix, (size_t)N, threads, out);
}
