// Preconditioners whose kernels live in files not yet added to the build.
#include "b2s_internal.cuh"

namespace b2s {
std::unique_ptr<PcImpl> make_pc_learned_ic0(b2s_ctx*, const CsrDev&, const b2s_pc_opts&) { fail(B2S_UNSUPPORTED, "learned IC(0) not built"); }
}
