// Preconditioners whose kernels live in files not yet added to the build.
#include "b2s_internal.cuh"

namespace b2s {
std::unique_ptr<PcImpl> make_pc_ic0(b2s_ctx*, const CsrDev&, const b2s_pc_opts&) { fail(B2S_UNSUPPORTED, "IC(0) not built"); }
std::unique_ptr<PcImpl> make_pc_ilu0(b2s_ctx*, const CsrDev&, const b2s_pc_opts&) { fail(B2S_UNSUPPORTED, "ILU(0) not built"); }
std::unique_ptr<PcImpl> make_pc_ssor(b2s_ctx*, const CsrDev&, const b2s_pc_opts&) { fail(B2S_UNSUPPORTED, "SSOR not built"); }
std::unique_ptr<PcImpl> make_pc_amg_csr(b2s_ctx*, const CsrDev&, const b2s_pc_opts&) { fail(B2S_UNSUPPORTED, "AMG not built"); }
std::unique_ptr<PcImpl> make_pc_amg_baij(b2s_ctx*, const BaijDev&, const b2s_pc_opts&) { fail(B2S_UNSUPPORTED, "AMG not built"); }
std::unique_ptr<PcImpl> make_pc_bilu0(b2s_ctx*, const BaijDev&, const b2s_pc_opts&) { fail(B2S_UNSUPPORTED, "block ILU(0) not built"); }
std::unique_ptr<PcImpl> make_pc_learned_ic0(b2s_ctx*, const CsrDev&, const b2s_pc_opts&) { fail(B2S_UNSUPPORTED, "learned IC(0) not built"); }
}
