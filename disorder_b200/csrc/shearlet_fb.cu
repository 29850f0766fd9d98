// Register-FFT shearlet passes of 88-, 64- and 44-point lines.
#include "shearlet.cuh"

namespace shl {

bool sh_fast_b(disorder_ctx_s* ctx, const ShArgs& a, int kind) {
  switch (a.N[a.axis]) {
    case 88: return sh_fast_launch<8, 11>(ctx, a, kind);
    case 64: return sh_fast_launch<8, 8>(ctx, a, kind);
    case 44: return sh_fast_launch<4, 11>(ctx, a, kind);
    default: return false;
  }
}

}  // namespace shl
