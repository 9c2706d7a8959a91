// ref_alias_shim.cpp — TEST INFRASTRUCTURE ONLY.
//
// Exposes the reference's own AliasTable (src/pathtracing/alias_table.h:19-79
// of ray847/CrystalGraphics, compiled unmodified from the read-only reference
// tree) through a C function, so tests can pin the oracle's restatement and
// the library's builder against it bit for bit.  Built by oracle/Makefile into
// oracle/_ref/libref_alias.so, only where the reference tree is present.
#include <cstdint>
#include <cstring>
#include <vector>

#include "src/pathtracing/alias_table.h"

extern "C" int ref_alias_build(const double* weights, uint32_t count, uint32_t* alias_out,
                               float* prob_out) {
  std::vector<double> w(weights, weights + count);
  crystal::graphics::AliasTable table(w);
  const auto& e = table.Data();
  if (e.size() != count) return -1;
  for (uint32_t i = 0; i < count; ++i) {
    alias_out[i] = e[i].alias;
    prob_out[i] = e[i].prob;
  }
  return 0;
}

// The reference's entries are value-initialised by vector::resize; report the
// raw bytes too so a zero-weight table can be compared exactly.
extern "C" int ref_alias_build_raw(const double* weights, uint32_t count, void* out) {
  std::vector<double> w(weights, weights + count);
  crystal::graphics::AliasTable table(w);
  const auto& e = table.Data();
  std::memcpy(out, e.data(), e.size() * sizeof(e[0]));
  return static_cast<int>(e.size());
}
