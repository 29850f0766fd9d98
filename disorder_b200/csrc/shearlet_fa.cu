// Register-FFT shearlet passes of 256-, 176- and 128-point lines.
#include "shearlet.cuh"

namespace shl {

bool sh_fast_a(disorder_ctx_s* ctx, const ShArgs& a, int kind) {
  switch (a.N[a.axis]) {
    case 256: return sh_fast_launch<16, 16>(ctx, a, kind);
    case 176: return sh_fast_launch<16, 11>(ctx, a, kind);
    case 128: return sh_fast_launch<16, 8>(ctx, a, kind);
    default: return false;
  }
}

}  // namespace shl
