// runs_check.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Calls the library's host-side run finder (kgctx::scan_gather, in
// supergwas_b200/csrc/capi.cpp) on caller rows and returns what the
// host-to-device pipeline would send: the runs' first rows and lengths, and
// the gathered rows in device order (the staging slices back to back).
#include <cstring>
#include <vector>

#include "../../supergwas_b200/csrc/ctx.hpp"

extern "C" uint64_t runs_check(const uint64_t* x, uint64_t s0, uint64_t cnt, uint32_t wpk, const uint64_t* bounds,
                               int n_bounds, uint64_t* first_out, uint32_t* len_out, uint64_t* rows_out) {
  std::vector<unsigned long long> bd(bounds, bounds + n_bounds);
  std::vector<uint64_t> stage((size_t)cnt * wpk);
  std::vector<uint64_t> first{7};  // entries already in the lists are kept
  std::vector<uint32_t> len{7};
  std::vector<kgctx::StageSeg> segs;
  const uint64_t nu = kgctx::scan_gather(x, s0, cnt, wpk, stage.data(), bd, first, len, segs);
  if (first.size() != nu + 1 || len.size() != nu + 1 || first[0] != 7 || len[0] != 7) return ~0ull;
  std::memcpy(first_out, first.data() + 1, nu * 8);
  std::memcpy(len_out, len.data() + 1, nu * 4);
  uint64_t d = 0;
  for (const auto& g : segs) {
    std::memcpy(rows_out + d * wpk, stage.data() + g.stage_row * wpk, g.rows * wpk * 8);
    d += g.rows;
  }
  return d == nu ? nu : ~0ull;
}
