// state.cu -- per-walker estimators from the evaluateGL arrays, and
// checkpoint / restore of a batch's walker state.
#include "common.cuh"
#include "host_api.hpp"

#include <cstring>

namespace qmc
{
// local kinetic energy -1/2 sum_i (L_i + |G_i|^2) of each walker, from the
// G and L of the last evaluateGL (WaveFunction.cpp:261-279): the Laplacian
// of psi over psi is L + G.G with G = grad log psi, L = lap log psi
__global__ void __launch_bounds__(256) kinetic_kernel(const double* __restrict__ G, const double* __restrict__ L,
                                                      int N, double* __restrict__ out)
{
  __shared__ double red[32];
  __shared__ double sum;
  const int w = blockIdx.x;
  const double* g = G + (size_t)w * N * 3;
  const double* l = L + (size_t)w * N;
  double s = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x)
    s += l[i] + g[3 * i] * g[3 * i] + g[3 * i + 1] * g[3 * i + 1] + g[3 * i + 2] * g[3 * i + 2];
  double v[1] = {s};
  block_sum<1>(v, red, &sum);
  if (threadIdx.x == 0)
    out[w] = -0.5 * sum;
}
} // namespace qmc

using namespace qmc;

namespace
{
// the persistent state of a batch: everything a later step reads; scratch
// (move rows, flush tiles, the FP64 inverse workspace, random numbers of a
// substep) is left out
struct Field
{
  void* p;
  size_t bytes;
};
std::vector<Field> state_fields(qmc_walkers* w)
{
  const DevWalkers& d = w->dw;
  const size_t W = d.W, N = d.N, Np = d.Npad, n = d.n, np = d.npad, k = d.k, es = w->fp32 ? 4 : 8;
  std::vector<Field> f = {{d.R, W * N * 3 * 8},         {d.Rs, W * 3 * Np * es},        {d.Ainv, W * 2 * n * np * es},
          {d.dpsiM, W * 6 * n * np * es}, {d.d2psiM, W * 2 * n * np * es}, {d.U, W * 2 * k * np * es},
          {d.V, W * 2 * k * np * es},    {d.Binv, W * 2 * k * k * 8},    {d.delay_list, W * 2 * k * 4},
          {d.delay_count, W * 2 * 4},    {d.det_log, W * 2 * 8},         {d.det_phase, W * 2 * 8},
          {d.j1_Vat, W * N * es},        {d.j1_Lap, W * N * es},         {d.j1_Grad, W * 3 * N * es},
          {d.j2_Uat, W * N * es},        {d.j2_d2Uat, W * N * es},       {d.j2_dUat, W * 3 * N * es},
          {d.j_log, W * 3 * 8},          {d.mt, W * (MT_N + 1) * 4},     {d.ms, W * sizeof(MoveState)},
          {d.G, W * N * 3 * 8},          {d.L, W * N * 8},               {d.logpsi, W * 8},
          {d.accepted, W * 8}};
  if (d.j3_cnt)
  {
    const size_t I = d.I;
    f.push_back({d.j3_Uat, W * N * es});
    f.push_back({d.j3_d2Uat, W * N * es});
    f.push_back({d.j3_dUat, W * 3 * N * es});
    f.push_back({d.j3_cnt, W * 2 * I * 4});
    f.push_back({d.j3_list, W * 2 * I * d.j3_cap * 4});
  }
  return f;
}

struct Header
{
  char magic[8];
  int version, W, N, n, npad, k, fp32, pad;
  int64_t steps_done, nlpp_calls;
  uint64_t payload;
};

Header make_header(qmc_walkers* w)
{
  Header h{};
  std::memcpy(h.magic, "QMCWALK", 8);
  h.version = 2, h.W = w->dw.W, h.N = w->dw.N, h.n = w->dw.n, h.npad = w->dw.npad, h.k = w->dw.k;
  h.fp32 = w->fp32 ? 1 : 0;
  h.steps_done = w->steps_done, h.nlpp_calls = w->nlpp_calls;
  h.payload = 0;
  for (auto& f : state_fields(w))
    h.payload += f.bytes;
  return h;
}
} // namespace

extern "C" {

int qmc_local_kinetic(qmc_walkers* w, double* kinetic)
{
  if (!w || !kinetic)
    return fail(QMC_ERR_ARG, "null pointer");
  const size_t W = w->dw.W;
  double* d = nullptr;
  CK(cudaMallocAsync(&d, W * sizeof(double), w->stream));
  kinetic_kernel<<<W, 256, 0, w->stream>>>(w->dw.G, w->dw.L, w->dw.N, d);
  CK(cudaGetLastError());
  w->launches++;
  CK(cudaMemcpyAsync(kinetic, d, W * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaFreeAsync(d, w->stream));
  CK(cudaStreamSynchronize(w->stream));
  return QMC_OK;
}

int qmc_walkers_checkpoint_bytes(qmc_walkers* w, size_t* bytes)
{
  if (!w || !bytes)
    return fail(QMC_ERR_ARG, "null pointer");
  *bytes = sizeof(Header) + make_header(w).payload;
  return QMC_OK;
}

int qmc_walkers_checkpoint(qmc_walkers* w, void* buffer, size_t bytes)
{
  if (!w || !buffer)
    return fail(QMC_ERR_ARG, "null pointer");
  const Header h = make_header(w);
  if (bytes < sizeof(Header) + h.payload)
    return fail(QMC_ERR_ARG, "checkpoint buffer too small (qmc_walkers_checkpoint_bytes)");
  unsigned char* p = static_cast<unsigned char*>(buffer);
  std::memcpy(p, &h, sizeof(h));
  p += sizeof(h);
  for (auto& f : state_fields(w))
  {
    CK(cudaMemcpyAsync(p, f.p, f.bytes, cudaMemcpyDeviceToHost, w->stream));
    p += f.bytes;
  }
  CK(cudaStreamSynchronize(w->stream));
  return QMC_OK;
}

int qmc_walkers_restore(qmc_walkers* w, const void* buffer, size_t bytes)
{
  if (!w || !buffer || bytes < sizeof(Header))
    return fail(QMC_ERR_ARG, "bad checkpoint buffer");
  Header h;
  std::memcpy(&h, buffer, sizeof(h));
  const Header mine = make_header(w);
  if (std::memcmp(h.magic, "QMCWALK", 8) || h.version != 2 || h.W != mine.W || h.N != mine.N || h.n != mine.n ||
      h.npad != mine.npad || h.k != mine.k || h.fp32 != mine.fp32 || h.payload != mine.payload ||
      bytes < sizeof(Header) + h.payload)
    return fail(QMC_ERR_ARG, "checkpoint does not match this batch (system, walkers, delay rank, precision)");
  const unsigned char* p = static_cast<const unsigned char*>(buffer) + sizeof(Header);
  for (auto& f : state_fields(w))
  {
    CK(cudaMemcpyAsync(f.p, p, f.bytes, cudaMemcpyHostToDevice, w->stream));
    p += f.bytes;
  }
  CK(cudaStreamSynchronize(w->stream));
  w->steps_done = h.steps_done;
  w->nlpp_calls = h.nlpp_calls;
  return QMC_OK;
}

} // extern "C"
