// tcgen05 tensor-core relight path (BF16 operands, FP32 accumulation in TMEM).
// Placeholder until the kernel lands: reports the path as unsupported.
#include "nwprt_internal.cuh"

namespace nwprt {

bool relight_tc_supported(const NetDims&, std::string* why) {
  if (why) *why = "tensor-core path not built";
  return false;
}
size_t tc_weight_bytes(const NetDims&) { return 0; }
void pack_tc_weights(const NetDims&, const float*, const float*, std::vector<uint16_t>* out) { out->clear(); }
size_t tc_env_table_bytes(const NetDims&, int) { return 0; }
void launch_tc_env_table(const NetDims&, const uint16_t*, const float*, int, uint16_t*, cudaStream_t) {
  fail(NWPRT_UNSUPPORTED, "tensor-core path not built");
}
void launch_relight_tc(const NetDims&, const HashLevels&, const float*, const uint16_t*, const TcJob*, int,
                       TcJob*, int, int, uint32_t*, cudaStream_t) {
  fail(NWPRT_UNSUPPORTED, "tensor-core path not built");
}

}  // namespace nwprt
