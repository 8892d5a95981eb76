// Test harness: the root search's period/mode chain (chain_advance in
// jdsurfg_b200/csrc/swdk_core.cuh) compiled for the host with the same
// production secular functions, one layered model's chain at a time, with
// or without bracket proposals, so CPU tests can plant proposals anywhere
// and check that none of them moves a root.  Built by
// tests/test_chain_host.py.
#include <cmath>
#include <vector>

#include <vector_types.h>  // float2 / float4 of the CUDA headers (plain host structs)

#include "swdk_core.cuh"

using namespace swdk;

// The flattened REAL*4 layer model (d, a, b, rho) top-down, the last layer
// the half-space; iwave 1 Love, 2 Rayleigh; nper periods, modes 1..nmode;
// cc the scan start, betmx the largest shear velocity.  prop (optional):
// (c, half-width) per slot, slot (mode m, period k) at (m - 1) * nper +
// k - 1, as the engine's proposal array holds them.  Writes the REAL*4
// roots and statuses of every slot and the chain's evaluation and proposal
// counts; returns the chain's ierr.
extern "C" int chain_host_run(int L, const float* d, const float* a, const float* b, const float* rho, int iwave,
                              int nper, const double* periods, int nmode, double cc, float betmx, const float* prop,
                              double* roots, int* status, long long* nevals, int* nprop_ok, int* nprop_fail) {
  if (L < 2 || nper < 1 || nper > KMAX_CHAIN || nmode < 1 || nmode * nper > KMAX_CHAIN) return -1;
  std::vector<float4> lay(L);
  for (int m = 0; m < L; ++m) lay[layer_index(L - 1 - m, 1, 0, L)] = float4{d[m], a[m], b[m], rho[m]};
  LayerView V{};
  V.lay = lay.data();
  V.fast = 1;
  V.ncol = 1;
  V.col = 0;
  V.lstride = L;
  V.L = L;
  V.llw = 1;
  V.nodes = nullptr;
  V.dl = nullptr;
  V.wave = iwave;
  ChainParams P{};
  P.t = periods;
  P.kmax = (int16_t)nper;
  P.nmode = (int16_t)nmode;
  P.igr = 0;
  P.iwave = (int8_t)iwave;
  P.refine = 1;
  P.rtol = 1e-10;
  P.sngl = 1;
  P.cc = cc;
  P.betmx = betmx;
  P.retry = RETRY_NONE;
  std::vector<double> cbuf(KMAX_CHAIN), cbbuf(KMAX_CHAIN + 24);
  std::vector<float2> pr;
  ChainIO io{};
  io.c = cbuf.data();
  io.cb = cbbuf.data();
  io.out = roots;
  io.stride = nper;
  io.ostride = 1;
  io.st = status;
  io.prop = nullptr;
  if (prop) {
    pr.resize((size_t)nmode * nper);
    for (size_t i = 0; i < pr.size(); ++i) pr[i] = float2{prop[2 * i], prop[2 * i + 1]};
    io.prop = pr.data();
  }
  for (int i = 0; i < nmode * nper; ++i) status[i] = -1;
  ChainState s;
  run_chain(V, P, io, s, true);
  *nevals = s.nevals;
  *nprop_ok = s.nprop_ok;
  *nprop_fail = s.nprop_fail;
  return s.ierr;
}
