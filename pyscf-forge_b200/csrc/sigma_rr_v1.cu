// Tile-shape variant 1 of the register-resident sigma kernel: 8 output
// rows per warp, 4 n-tiles of 8 columns per tile (one translation unit per
// variant so that the instances compile in parallel).
#include "sigma_rr_kernel.cuh"

namespace csffci {

int rr_dispatch_v1(int norb, RRArgs& g, size_t smem, cudaStream_t stream) {
#define RR(K, W) return launch_rr<K, W, 8, 4>(g, smem, stream)
  switch (norb) {
    case 4: RR(3, 2);
    case 5: RR(4, 2);
    case 6: RR(6, 3);
    case 7: RR(7, 4);
    case 8: RR(9, 5);
    case 9: RR(12, 6);
    case 10: RR(14, 7);
    case 11: RR(17, 9);
    case 12: RR(20, 10);
    case 13: RR(23, 12);
    case 14: RR(27, 14);
    case 15: RR(30, 15);
    case 16: RR(34, 17);
    default:
      break;
  }
#undef RR
  set_error("sigma: no tile variant 1 instance for norb=%d", norb);
  return CSFFCI_ERR_INVALID;
}

}  // namespace csffci
