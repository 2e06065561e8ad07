// Tile-shape variant 2 of the register-resident sigma kernel: 16 output
// rows per warp, 2 n-tiles of 8 columns per tile (one translation unit per
// variant so that the instances compile in parallel).
#include "sigma_rr_kernel.cuh"

namespace csffci {

int rr_dispatch_v2(int norb, RRArgs& g, size_t smem, cudaStream_t stream) {
#define RR(K, W) return launch_rr<K, W, 16, 2>(g, smem, stream)
  switch (norb) {
    case 4: RR(3, 1);
    case 5: RR(4, 1);
    case 6: RR(6, 2);
    case 7: RR(7, 2);
    case 8: RR(9, 3);
    case 9: RR(12, 3);
    case 10: RR(14, 4);
    case 11: RR(17, 5);
    case 12: RR(20, 5);
    case 13: RR(23, 6);
    case 14: RR(27, 7);
    case 15: RR(30, 8);
    case 16: RR(34, 9);
    default:
      break;
  }
#undef RR
  set_error("sigma: no tile variant 2 instance for norb=%d", norb);
  return CSFFCI_ERR_INVALID;
}

}  // namespace csffci
