// api.cu -- the C ABI (include/qmcgpu.h): handles, device memory, launches.
//
// Host side of the drop-in boundary.  Every entry point returns a status and
// records a message retrievable with qmc_last_error(); nothing here exits the
// process.  All compute runs in the kernels of sweep.cu / others.cu; there
// is no host fallback for any hot-path operation.
#include "host_api.hpp"
#include "host_lattice.hpp"
#include "tc.cuh"

#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

using namespace qmc;

thread_local std::string g_err;

int fail(int code, const std::string& msg)
{
  g_err = msg;
  return code;
}

// set while walkers_footprint sizes a batch: dalloc only counts bytes
static thread_local bool g_dry = false;
// set while a request-loop job's walkers are allocated: dalloc takes the
// memory stream-ordered from the server's pool on its stream (no device-wide
// synchronisation, memory reused without returning it to the driver)
static thread_local cudaStream_t g_alloc_stream = nullptr;
static thread_local cudaMemPool_t g_alloc_pool  = nullptr;
struct AllocScope
{
  cudaStream_t s0;
  cudaMemPool_t p0;
  AllocScope(cudaStream_t s, cudaMemPool_t p) : s0(g_alloc_stream), p0(g_alloc_pool)
  {
    g_alloc_stream = s;
    g_alloc_pool   = p;
  }
  ~AllocScope()
  {
    g_alloc_stream = s0;
    g_alloc_pool   = p0;
  }
};

template <typename P> static int dalloc(std::vector<void*>& list, size_t& bytes, P** p, size_t count)
{
  *p = nullptr;
  if (count == 0)
    count = 1;
  if (g_dry)
  {
    bytes += count * sizeof(P);
    return QMC_OK;
  }
  cudaError_t e = g_alloc_stream
      ? cudaMallocFromPoolAsync((void**)p, count * sizeof(P), g_alloc_pool, g_alloc_stream)
      : cudaMalloc((void**)p, count * sizeof(P));
  if (e != cudaSuccess)
    return fail(QMC_ERR_OOM, std::string("device allocation failed: ") + cudaGetErrorString(e));
  e = g_alloc_stream ? cudaMemsetAsync(*p, 0, count * sizeof(P), g_alloc_stream) : cudaMemset(*p, 0, count * sizeof(P));
  if (e != cudaSuccess)
    return fail(QMC_ERR_CUDA, cudaGetErrorString(e));
  list.push_back((void*)*p);
  bytes += count * sizeof(P);
  return QMC_OK;
}

int device_status(qmc_walkers* w)
{
  unsigned st = 0;
  CK(cudaMemcpyAsync(&st, w->dw.status, sizeof(unsigned), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaStreamSynchronize(w->stream));
  if (st)
    CK(cudaMemsetAsync(w->dw.status, 0, sizeof(unsigned), w->stream));
  return status_from_bits(st);
}

int status_from_bits(unsigned st)
{
  if (st)
  {
    if (st & DEV_ERR_SINGULAR)
      return fail(QMC_ERR_SINGULAR, "zero pivot in the FP64 inverse of a Slater matrix");
    if (st & DEV_ERR_NONFINITE)
      return fail(QMC_ERR_NONFINITE, "non-finite wavefunction ratio");
    if (st & DEV_ERR_TIMEOUT)
      return fail(QMC_ERR_TIMEOUT, "a bounded wait on the tensor-core pipeline gave up");
    if (st & DEV_ERR_STATE)
      return fail(QMC_ERR_STATE, "move protocol violated (no proposed move for this electron)");
    if (st & DEV_ERR_CAPACITY)
      return fail(QMC_ERR_CAPACITY, "a J3 electron list of an ion, the ions near one position or the "
                                    "pairs of one move exceeded its fixed capacity");
    return fail(QMC_ERR_CUDA, "device error bits set");
  }
  return QMC_OK;
}

extern "C" {

const char* qmc_status_string(int s)
{
  switch (s)
  {
  case QMC_OK: return "QMC_OK";
  case QMC_ERR_ARG: return "QMC_ERR_ARG";
  case QMC_ERR_CUDA: return "QMC_ERR_CUDA";
  case QMC_ERR_OOM: return "QMC_ERR_OOM";
  case QMC_ERR_SINGULAR: return "QMC_ERR_SINGULAR";
  case QMC_ERR_NONFINITE: return "QMC_ERR_NONFINITE";
  case QMC_ERR_TIMEOUT: return "QMC_ERR_TIMEOUT";
  case QMC_ERR_STATE: return "QMC_ERR_STATE";
  case QMC_ERR_NODEVICE: return "QMC_ERR_NODEVICE";
  case QMC_ERR_ADMISSION: return "QMC_ERR_ADMISSION";
  case QMC_ERR_CAPACITY: return "QMC_ERR_CAPACITY";
  default: return "QMC_ERR_UNKNOWN";
  }
}
const char* qmc_last_error(void) { return g_err.c_str(); }

int qmc_init(int device)
{
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
    return fail(QMC_ERR_NODEVICE, "no CUDA device");
  if (device < 0 || device >= n)
    return fail(QMC_ERR_ARG, "device index out of range");
  CK(cudaSetDevice(device));
  cudaDeviceProp p;
  CK(cudaGetDeviceProperties(&p, device));
  if (p.major != 10)
    return fail(QMC_ERR_NODEVICE, "library built for sm_100a; device is sm_" + std::to_string(p.major) +
                                      std::to_string(p.minor));
  return QMC_OK;
}

// -------------------------------------------------------------- builders --
int qmc_nio_count(int cell, int na, int nb, int nc, int* n_ions)
{
  if (!n_ions || na < 1 || nb < 1 || nc < 1)
    return fail(QMC_ERR_ARG, "bad tiling");
  *n_ions = (cell == QMC_NIO_REF32 ? 32 : 4) * na * nb * nc;
  return QMC_OK;
}
int qmc_nio_build(int cell, int na, int nb, int nc, int quirks, double* lattice, double* ion_pos, int* ion_group,
                  int* n_groups, double* spo_lattice)
{
  if (!lattice || !ion_pos || !ion_group || !n_groups || !spo_lattice || na < 1 || nb < 1 || nc < 1)
    return fail(QMC_ERR_ARG, "bad arguments to qmc_nio_build");
  qmc_host::Ions s = cell == QMC_NIO_REF32 ? qmc_host::nio_ref32(na, nb, nc, quirks) : qmc_host::nio_prim4(na, nb, nc);
  std::memcpy(lattice, s.lattice, sizeof(s.lattice));
  std::memcpy(spo_lattice, s.spo_lattice, sizeof(s.spo_lattice));
  std::copy(s.pos.begin(), s.pos.end(), ion_pos);
  std::copy(s.group.begin(), s.group.end(), ion_group);
  *n_groups = s.n_groups;
  return QMC_OK;
}
int qmc_functor_setup(int n_params, double rcut, double cusp, const double* params, qmc_functor* out)
{
  int st = qmc_host::functor_setup(n_params, rcut, cusp, params, out);
  return st ? fail(st, "bad functor parameters") : QMC_OK;
}
int qmc_lattice_ws_radius(const double* lattice, double* ws)
{
  if (!lattice || !ws)
    return fail(QMC_ERR_ARG, "null pointer");
  *ws = qmc_host::ws_radius(lattice);
  return QMC_OK;
}
int qmc_nio_jastrows(const double* lattice, qmc_functor* j1_O, qmc_functor* j1_Ni, qmc_functor* j2_uu,
                     qmc_functor* j2_ud)
{
  if (!lattice || !j1_O || !j1_Ni || !j2_uu || !j2_ud)
    return fail(QMC_ERR_ARG, "null pointer");
  const double ws       = qmc_host::ws_radius(lattice);
  const double Yuu[10]  = {0.3062333936,  0.2068358231,  0.1324267459,  0.08673342451,  0.05641590391,
                          0.03626533946, 0.02269217959, 0.01331043612, 0.006750919735, 0.002827476478};
  const double Yud[10]  = {0.4397856796,  0.2589475889,  0.1516634434,  0.08962897215, 0.05676614496,
                          0.03675758961, 0.02294244601, 0.01343860721, 0.00681803725, 0.002864695148};
  const double YO[10]   = {-1.060468469,   -0.9741652012,  -0.8785027166, -0.6350075366,  -0.3276892194,
                         -0.08646817952, -0.07340983171, -0.0377479213, -0.01507835571, -0.001101691898};
  const double YNi[10]  = {-3.058259288,  -3.077898004,  -2.51188807,   -1.570208063,  -0.6204423266,
                          0.06272826611, 0.06228214399, 0.06665099211, 0.03230352443, 0.009254036239};
  const double rc2 = std::min(ws, 5.5727792532), rc1 = std::min(ws, 4.8261684030);
  qmc_host::functor_setup(10, rc2, 0.0, Yuu, j2_uu);
  qmc_host::functor_setup(10, rc2, 0.0, Yud, j2_ud);
  qmc_host::functor_setup(10, rc1, -0.25, YO, j1_O);
  qmc_host::functor_setup(10, rc1, -0.25, YNi, j1_Ni);
  return QMC_OK;
}

int qmc_j3_functor_setup(double rcut, const double* params, qmc_j3_functor* out)
{
  int st = qmc_host::j3_functor_setup(rcut, params, out);
  return st ? fail(st, "bad three-body functor parameters") : QMC_OK;
}
// buildJeeI (nio.hpp:171-245): the four PolynomialFunctor3D parameter sets
// of the reference's NiO input, in the order it adds them
int qmc_nio_j3(const double* lattice, qmc_j3_functor* same, qmc_j3_functor* diff)
{
  if (!lattice || !same || !diff)
    return fail(QMC_ERR_ARG, "null pointer");
  static const double Y[4][QMC_J3_PARAMS] = {
      {-0.003356164484, 0.002412623253, 0.01653623839, 0.0008341346169, -0.002808360734, 0.000710697475,
       0.01076942152, 0.0009228283355, 0.01576022161, -0.003585259096, 0.003323106938, -0.02282975998,
       -0.002246144403, -0.007196992871, -0.00404316239, 0.001465337212, 0.02026982926, -0.03528735393,
       0.04594087928, -0.008776410679, -0.001552528476, -0.005554407743, 0.001858594451, 0.002001634408,
       0.0009302256139, -0.0006304447229},
      {-0.006861627197, 0.003278047306, 0.03324006545, 0.003097361067, -0.004710623571, 9.652180317e-06,
       0.02212708787, -0.003718893286, 0.03390124932, -0.00710566395, 0.008807743592, -0.04281661568,
       -0.008463011294, -0.01269994613, -0.002005229447, 0.002186590944, 0.03350196472, -0.05677253817,
       0.07810604648, -0.009629896208, -0.006372643712, -0.01056861605, 0.002485188615, 0.008392442289,
       1.073423014e-05, -0.0004812466328},
      {-0.003775082438, -0.00169971229, 0.02162925441, 0.005674020544, -0.0008296047161, 0.00128057705,
       0.005487203215, 0.001637322446, 0.02976838198, -0.0003207100945, 0.01143855436, -0.05336741304,
       -0.00732359381, -0.01556942626, 0.0001149478453, 0.001838601199, 0.02570154203, -0.0675325214,
       0.1080671614, -0.01258358969, 0.001839834045, -0.02422400426, 0.005154953014, 0.003510582598,
       0.007464427016, -0.002454817757},
      {-0.009590393593, 0.002498010871, 0.04225872633, 0.00460311261, -0.01071033503, 0.001253155062,
       0.02934351285, -0.01823794726, 0.07224890393, -0.01020046849, 0.006310807929, -0.05655009412,
       -0.0363775247, 0.002062411388, 0.02037856173, 0.003372676617, 0.03915277249, -0.02680556816,
       0.08648136635, 0.01499088063, -0.02231984329, -0.02399792096, 0.001105720128, 0.02196005181,
       0.003162638982, -0.00119645772}};
  const double rcut = std::min(qmc_host::ws_radius(lattice), 4.8261684030);
  for (int sp = 0; sp < 2; ++sp)
  {
    qmc_host::j3_functor_setup(rcut, Y[2 * sp], same + sp);
    qmc_host::j3_functor_setup(rcut, Y[2 * sp + 1], diff + sp);
  }
  return QMC_OK;
}

// The synthetic Jastrows of the NiO workloads: n_params knot values per
// functor, uniform in [-0.1, 0.1) from SplitMix64(seed, 64*f + i) with
// f = 0 (uu), 1 (ud), 2.. (one per ion species); cutoff = half the
// Wigner-Seitz radius; cusp 0 (J2) and -0.25 (J1) as the reference tables.
int qmc_synthetic_jastrows(const double* lattice, int n_groups, uint64_t seed, int n_params, qmc_functor* j1,
                           qmc_functor* j2_uu, qmc_functor* j2_ud)
{
  if (!lattice || !j1 || !j2_uu || !j2_ud || n_groups < 1 || n_groups > QMC_MAX_ION_GROUPS || n_params < 2 ||
      n_params + 4 > QMC_MAX_FUNCTOR_COEFS)
    return fail(QMC_ERR_ARG, "bad synthetic Jastrow arguments");
  const double rc = 0.5 * qmc_host::ws_radius(lattice);
  double k[QMC_MAX_FUNCTOR_COEFS];
  auto knots = [&](int f) {
    for (int i = 0; i < n_params; ++i)
      k[i] = 0.2 * splitmix_uniform(seed, 64ull * f + i) - 0.1;
  };
  knots(0);
  qmc_host::functor_setup(n_params, rc, 0.0, k, j2_uu);
  knots(1);
  qmc_host::functor_setup(n_params, rc, 0.0, k, j2_ud);
  for (int g = 0; g < n_groups; ++g)
  {
    knots(2 + g);
    qmc_host::functor_setup(n_params, rc, -0.25, k, &j1[g]);
  }
  return QMC_OK;
}

} // extern "C"

// --------------------------------------------------------------- system --
template <typename T>
__global__ void fill_table_kernel(T* coefs, size_t n_points, int norb, int npad, int mode, uint64_t seed,
                                  const double* field, const double* pref, const double* user)
{
  const size_t total = n_points * (size_t)npad;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x)
  {
    const size_t g = e / npad;
    const int j    = (int)(e % npad);
    double v       = 0.0;
    if (j < norb)
    {
      if (mode == QMC_FILL_UNIFORM)
        v = splitmix_uniform(seed, g * norb + j) - 0.5;
      else if (mode == QMC_FILL_UNIFORM_F32)
        v = (double)(float)(splitmix_uniform(seed, g * norb + j) - 0.5);
      else if (mode == QMC_FILL_REFERENCE)
        v = field[g] * pref[j];
      else
        v = user[g * norb + j];
    }
    coefs[e] = (T)v;
  }
}

extern "C" {

int qmc_system_create(const qmc_system_desc* d, int precision, qmc_system** out)
{
  if (!d || !out)
    return fail(QMC_ERR_ARG, "null pointer");
  *out           = nullptr;
  const int comp = d->components ? d->components : QMC_WF_ALL;
  if (d->n_elec <= 0 || d->n_up < 0 || d->n_orb <= 0 || d->n_ions <= 0 || d->n_ion_groups < 1 ||
      d->n_ion_groups > QMC_MAX_ION_GROUPS || d->grid[0] < 1 || d->grid[1] < 1 || d->grid[2] < 1 || !d->ion_pos ||
      !d->ion_group)
    return fail(QMC_ERR_ARG, "bad system description");
  if ((comp & QMC_WF_DET) && (d->n_up != d->n_orb || d->n_elec - d->n_up != d->n_orb))
    return fail(QMC_ERR_ARG, "the determinants need n_up == n_elec - n_up == n_orb");
  if (d->spo_fill < QMC_FILL_USER || d->spo_fill > QMC_FILL_UNIFORM_F32)
    return fail(QMC_ERR_ARG, "unknown spline fill");
  if (d->spo_fill == QMC_FILL_USER && !d->spo_user_coefs)
    return fail(QMC_ERR_ARG, "QMC_FILL_USER needs spo_user_coefs");
  for (int i = 1; i < d->n_ions; ++i)
    if (d->ion_group[i] < d->ion_group[i - 1])
      return fail(QMC_ERR_ARG, "ions must be grouped by species");
  if (comp & QMC_WF_J3)
    for (int g = 0; g < d->n_ion_groups; ++g)
      if (!(d->j3_same[g].cutoff > 0) || d->j3_same[g].cutoff != d->j3_diff[g].cutoff)
        // ThreeBodyJastrow::check_complete aborts on unequal radii
        return fail(QMC_ERR_ARG, "J3 functors of an ion species need one positive cutoff");
  auto* s  = new qmc_system_s;
  s->fp32  = precision == QMC_PREC_MIXED;
  DevSystem& h = s->h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.lattice, d->lattice, sizeof(h.lattice));
  qmc_host::bconds(d->lattice, h.rb, h.gb, h.corners);
  h.mi_scale2 = qmc_host::min_metric_eigenvalue(h.rb) * (1.0 - 1e-6);
  qmc_host::inverse3(d->spo_lattice, h.spoG);
  for (int k = 0; k < 3; ++k)
  {
    h.grid[k]          = d->grid[k];
    const double delta = (1.0 - 0.0) / (double)d->grid[k];
    h.dinv[k]          = 1.0 / delta;
  }
  h.norb         = d->n_orb;
  h.npad         = round_up(d->n_orb, 32);
  h.zs           = h.npad;
  h.ys           = (long long)(d->grid[2] + 3) * h.zs;
  h.xs           = (long long)(d->grid[1] + 3) * h.ys;
  h.table_fp32   = s->fp32 ? 1 : 0;
  h.n_ions       = d->n_ions;
  h.n_groups     = d->n_ion_groups;
  h.n_elec       = d->n_elec;
  h.n_up         = d->n_up;
  h.lap_mode     = d->lap_mode;
  h.comp         = comp;
  for (int g = 0; g < QMC_MAX_ION_GROUPS; ++g)
  {
    int f = -1, l = -1;
    for (int i = 0; i < d->n_ions; ++i)
      if (d->ion_group[i] == g)
      {
        if (f < 0)
          f = i;
        l = i + 1;
      }
    h.gfirst[g] = f < 0 ? 0 : f;
    h.glast[g]  = f < 0 ? 0 : l;
  }
  auto cp_functor = [](DevFunctor& o, const qmc_functor& f) {
    o.n      = f.n_coefs;
    o.cutoff = f.cutoff;
    o.dinv   = f.delta_r_inv;
    for (int c = 0; c < QMC_MAX_FUNCTOR_COEFS; ++c)
      o.c[c] = c < f.n_coefs ? f.coefs[c] : 0.0;
  };
  for (int g = 0; g < QMC_MAX_ION_GROUPS; ++g)
    cp_functor(h.j1[g], d->j1[g]);
  cp_functor(h.j2uu, d->j2_uu);
  cp_functor(h.j2ud, d->j2_ud);
  // functor index (int)(r * dinv) + 3 must stay inside the coefficient table
  // for r < cutoff: (numKnots-1) intervals + 3 < n_coefs holds by construction.
  int st = QMC_OK;
  const size_t npts = (size_t)(d->grid[0] + 3) * (d->grid[1] + 3) * (d->grid[2] + 3);
  const size_t elem = s->fp32 ? 4 : 8;
  void* coefs       = nullptr;
  cudaError_t e     = cudaMalloc(&coefs, npts * h.npad * elem);
  if (e != cudaSuccess)
  {
    delete s;
    return fail(QMC_ERR_OOM, "spline table allocation failed: " + std::string(cudaGetErrorString(e)));
  }
  s->allocs.push_back(coefs);
  s->bytes += npts * h.npad * elem;
  h.coefs      = coefs;
  h.coef_bytes = npts * h.npad * elem;
  double *d_field = nullptr, *d_pref = nullptr, *d_user = nullptr;
  if (d->spo_fill == QMC_FILL_REFERENCE)
  {
    std::mt19937 mt((uint32_t)d->spo_seed);
    std::uniform_real_distribution<double> uni;
    std::vector<double> field(npts), pref(d->n_orb);
    for (auto& f : field)
      f = uni(mt);
    for (int ind = 0; ind < d->n_orb; ind++)
      pref[ind] = std::cos(2 * M_PI * ind / d->n_orb);
    cudaMalloc(&d_field, npts * sizeof(double));
    cudaMalloc(&d_pref, d->n_orb * sizeof(double));
    cudaMemcpy(d_field, field.data(), npts * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(d_pref, pref.data(), d->n_orb * sizeof(double), cudaMemcpyHostToDevice);
  }
  else if (d->spo_fill == QMC_FILL_USER)
  {
    cudaMalloc(&d_user, npts * d->n_orb * sizeof(double));
    cudaMemcpy(d_user, d->spo_user_coefs, npts * d->n_orb * sizeof(double), cudaMemcpyHostToDevice);
  }
  if (s->fp32)
    fill_table_kernel<float><<<4 * 148, 256>>>((float*)coefs, npts, d->n_orb, h.npad, d->spo_fill, d->spo_seed,
                                              d_field, d_pref, d_user);
  else
    fill_table_kernel<double><<<4 * 148, 256>>>((double*)coefs, npts, d->n_orb, h.npad, d->spo_fill, d->spo_seed,
                                               d_field, d_pref, d_user);
  e = cudaDeviceSynchronize();
  cudaFree(d_field);
  cudaFree(d_pref);
  cudaFree(d_user);
  if (e != cudaSuccess)
  {
    for (void* p : s->allocs)
      cudaFree(p);
    delete s;
    return fail(QMC_ERR_CUDA, std::string("spline fill: ") + cudaGetErrorString(e));
  }
  // ions: AoS double + SoA in the walker precision
  double* ion_pos = nullptr;
  if ((st = dalloc(s->allocs, s->bytes, &ion_pos, 3 * (size_t)d->n_ions)))
    return st;
  cudaMemcpy(ion_pos, d->ion_pos, 3 * d->n_ions * sizeof(double), cudaMemcpyHostToDevice);
  h.ion_pos = ion_pos;
  std::vector<double> soa(3 * (size_t)d->n_ions);
  for (int i = 0; i < d->n_ions; ++i)
    for (int c = 0; c < 3; ++c)
      soa[(size_t)c * d->n_ions + i] = d->ion_pos[3 * i + c];
  if (s->fp32)
  {
    std::vector<float> f(soa.begin(), soa.end());
    float* p = nullptr;
    if ((st = dalloc(s->allocs, s->bytes, &p, f.size())))
      return st;
    cudaMemcpy(p, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice);
    h.ion_soa = p;
  }
  else
  {
    double* p = nullptr;
    if ((st = dalloc(s->allocs, s->bytes, &p, soa.size())))
      return st;
    cudaMemcpy(p, soa.data(), soa.size() * sizeof(double), cudaMemcpyHostToDevice);
    h.ion_soa = p;
  }
  if (comp & QMC_WF_J3)
  {
    // gammas in the walker precision, [species][same, opposite][64]
    std::vector<double> gm((size_t)QMC_MAX_ION_GROUPS * 2 * 64, 0.0);
    for (int g = 0; g < d->n_ion_groups; ++g)
    {
      h.j3_icut[g] = 0.5 * d->j3_same[g].cutoff;
      for (int q = 0; q < 64; ++q)
      {
        gm[(size_t)(2 * g) * 64 + q]     = d->j3_same[g].gamma[q];
        gm[(size_t)(2 * g + 1) * 64 + q] = d->j3_diff[g].gamma[q];
      }
    }
    void* p = nullptr;
    if ((st = dalloc(s->allocs, s->bytes, reinterpret_cast<unsigned char**>(&p), gm.size() * (s->fp32 ? 4 : 8))))
      return st;
    if (s->fp32)
    {
      std::vector<float> f(gm.begin(), gm.end());
      cudaMemcpy(p, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice);
    }
    else
      cudaMemcpy(p, gm.data(), gm.size() * sizeof(double), cudaMemcpyHostToDevice);
    h.j3_gamma = p;
  }
  if ((st = dalloc(s->allocs, s->bytes, &s->d, 1)))
    return st;
  CK(cudaMemcpy(s->d, &h, sizeof(DevSystem), cudaMemcpyHostToDevice));
  *out = s;
  return QMC_OK;
}

int qmc_system_destroy(qmc_system* s)
{
  if (!s)
    return QMC_OK;
  cudaDeviceSynchronize();
  for (void* p : s->allocs)
    cudaFree(p);
  delete s;
  return QMC_OK;
}
int qmc_system_bytes(const qmc_system* s, size_t* bytes)
{
  if (!s || !bytes)
    return fail(QMC_ERR_ARG, "null pointer");
  *bytes = s->bytes;
  return QMC_OK;
}

static int spo_points(qmc_system* s, int n_pos, const double* pos, double* v, double* g, double* h, bool vonly)
{
  if (!s || n_pos < 0 || (n_pos > 0 && !pos))
    return fail(QMC_ERR_ARG, "bad arguments");
  if (n_pos == 0)
    return QMC_OK;
  const int norb = s->h.norb;
  double *dp = nullptr, *dv = nullptr, *dg = nullptr, *dh = nullptr;
  CK(cudaMalloc(&dp, 3 * n_pos * sizeof(double)));
  CK(cudaMalloc(&dv, (size_t)n_pos * norb * sizeof(double)));
  CK(cudaMalloc(&dg, (size_t)n_pos * 3 * norb * sizeof(double)));
  CK(cudaMalloc(&dh, (size_t)n_pos * 6 * norb * sizeof(double)));
  CK(cudaMemcpy(dp, pos, 3 * n_pos * sizeof(double), cudaMemcpyHostToDevice));
  CK(launch_spo_points(s->fp32, s->d, n_pos, dp, dv, dg, dh, vonly, 0));
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess)
  {
    if (v)
      cudaMemcpy(v, dv, (size_t)n_pos * norb * sizeof(double), cudaMemcpyDeviceToHost);
    if (g && !vonly)
      cudaMemcpy(g, dg, (size_t)n_pos * 3 * norb * sizeof(double), cudaMemcpyDeviceToHost);
    if (h && !vonly)
      cudaMemcpy(h, dh, (size_t)n_pos * 6 * norb * sizeof(double), cudaMemcpyDeviceToHost);
  }
  cudaFree(dp);
  cudaFree(dv);
  cudaFree(dg);
  cudaFree(dh);
  CK(e);
  return QMC_OK;
}
int qmc_spo_evaluate_vgh(qmc_system* s, int n_pos, const double* pos, double* v, double* g, double* h)
{
  return spo_points(s, n_pos, pos, v, g, h, false);
}
int qmc_spo_evaluate_v(qmc_system* s, int n_pos, const double* pos, double* v)
{
  return spo_points(s, n_pos, pos, v, nullptr, nullptr, true);
}

// -------------------------------------------------------------- walkers --
static int alloc_walkers(qmc_walkers* w, qmc_system* s, int W, int k)
{
  DevWalkers& d = w->dw;
  const DevSystem& h = s->h;
  const size_t es = s->fp32 ? 4 : 8;
  d.W = W, d.N = h.n_elec, d.Npad = round_up(h.n_elec, 32), d.n = h.norb, d.npad = h.npad, d.I = h.n_ions, d.k = k;
  d.wait_cycles = kTcWaitCycles;
  const size_t N = d.N, Np = d.Npad, n = d.n, np = d.npad, KK = k;
  std::vector<void*>& L = w->allocs;
  size_t& B             = w->bytes;
  auto T = [&](void** p, size_t count) -> int {
    unsigned char* q = nullptr;
    int st           = dalloc(L, B, &q, count * es);
    *p               = q;
    return st;
  };
  int st = 0;
  st |= dalloc(L, B, &d.R, W * N * 3);
  st |= T(&d.Rs, W * 3 * Np);
  st |= T(&d.Ainv, W * 2 * n * np);
  st |= T(&d.dpsiM, W * 2 * 3 * n * np);
  st |= T(&d.d2psiM, W * 2 * n * np);
  st |= T(&d.U, W * 2 * KK * np);
  st |= T(&d.V, W * 2 * KK * np);
  st |= dalloc(L, B, &d.Binv, W * 2 * KK * KK);
  st |= dalloc(L, B, &d.delay_list, W * 2 * KK);
  st |= dalloc(L, B, &d.delay_count, W * 2);
  st |= dalloc(L, B, &d.det_log, W * 2);
  st |= dalloc(L, B, &d.det_phase, W * 2);
  st |= T(&d.j1_Vat, W * N);
  st |= T(&d.j1_Lap, W * N);
  st |= T(&d.j1_Grad, W * 3 * N);
  st |= T(&d.j2_Uat, W * N);
  st |= T(&d.j2_d2Uat, W * N);
  st |= T(&d.j2_dUat, W * 3 * N);
  st |= dalloc(L, B, &d.j_log, W * 3);
  d.j3_Uat = d.j3_d2Uat = d.j3_dUat = nullptr;
  d.j3_cnt = d.j3_list = nullptr;
  d.j3_cap = 0;
  if (h.comp & QMC_WF_J3)
  {
    d.j3_cap = j3_list_capacity(h.n_elec, h.n_up);
    st |= T(&d.j3_Uat, W * N);
    st |= T(&d.j3_d2Uat, W * N);
    st |= T(&d.j3_dUat, W * 3 * N);
    st |= dalloc(L, B, &d.j3_cnt, W * 2 * (size_t)d.I);
    st |= dalloc(L, B, &d.j3_list, W * 2 * (size_t)d.I * d.j3_cap);
  }
  st |= dalloc(L, B, &d.mt, W * (size_t)(MT_N + 1));
  st |= dalloc(L, B, &d.words, W * (8 * N + 8));
  st |= dalloc(L, B, &d.ur, W * N);
  st |= dalloc(L, B, &d.delta, W * 3 * N);
  st |= T(&d.invRow, W * EPOCH_MAX * np);
  st |= T(&d.psiV, W * np);
  st |= T(&d.dpsiV, W * 3 * np);
  st |= T(&d.d2psiV, W * np);
  st |= T(&d.U2, W * KK * np);
  st |= T(&d.tm, W * n * KK);
  st |= dalloc(L, B, &d.ms, W);
  st |= dalloc(L, B, &d.G, W * N * 3);
  st |= dalloc(L, B, &d.L, W * N);
  st |= dalloc(L, B, &d.logpsi, W);
  st |= dalloc(L, B, &d.accepted, W);
  st |= dalloc(L, B, &d.out_grad, W * 3);
  st |= dalloc(L, B, &d.out_ratio, W);
  st |= dalloc(L, B, &d.accept_flags, W);
  st |= dalloc(L, B, &d.status, 1);
  st |= dalloc(L, B, &w->d_task, 1);
  st |= dalloc(L, B, &w->d_displ, W * 3);
  st |= dalloc(L, B, &w->d_step, W * 4);
  st |= dalloc(L, B, &w->d_flags, W);
  d.lu = nullptr;
  if (st)
    return QMC_ERR_OOM;
  if (g_dry)
    return QMC_OK;
  // (dalloc has zeroed every array, stream-ordered for a pooled batch)
  if (!g_alloc_stream && d.j3_cnt)
  {
    CK(cudaMemset(d.j3_cnt, 0, W * 2 * (size_t)d.I * sizeof(int)));
    CK(cudaMemset(d.j3_Uat, 0, W * N * es));
    CK(cudaMemset(d.j3_d2Uat, 0, W * N * es));
    CK(cudaMemset(d.j3_dUat, 0, W * 3 * N * es));
  }
  if (!g_alloc_stream)
    CK(cudaMemset(d.j_log, 0, W * 3 * sizeof(double)));
  std::vector<MoveState> ms(W);
  for (auto& m : ms)
  {
    std::memset(&m, 0, sizeof(m));
    m.active       = -1;
    m.invrow_id[0] = m.invrow_id[1] = -1;
    m.partial[0] = m.partial[1] = 1;
    m.j_partial                 = 1;
  }
  if (g_alloc_stream) // pageable source: staged before the call returns
    CK(cudaMemcpyAsync(d.ms, ms.data(), W * sizeof(MoveState), cudaMemcpyHostToDevice, g_alloc_stream));
  else
    CK(cudaMemcpy(d.ms, ms.data(), W * sizeof(MoveState), cudaMemcpyHostToDevice));
  return QMC_OK;
}

} // extern "C"

size_t walkers_footprint(qmc_system* s, int W, int k)
{
  qmc_walkers_s t;
  t.sys  = s;
  t.fp32 = s->fp32;
  g_dry  = true;
  alloc_walkers(&t, s, W, k);
  g_dry = false;
  const int nvec    = s->h.npad / (s->fp32 ? 4 : 2);
  const int threads = std::min(256, std::max(std::max(64, 2 * k), round_up(nvec, 32)));
  size_t b          = t.bytes + (size_t)W * 2 * s->h.norb * s->h.npad * sizeof(double); // FP64 inverse scratch
  if (s->fp32 && threads >= 128 && k <= TC_KD && (s->h.comp & QMC_WF_DET))
    b += (size_t)W * tc_image_floats(s->h.npad, k) * sizeof(float);
  return b;
}

extern "C" {

static void free_walkers(qmc_walkers* w)
{
  if (w->alloc_stream)
  {
    // a pooled batch: its memory returns to the pool behind its last work
    // on the stream, without waiting for it
    for (void* p : w->allocs)
      cudaFreeAsync(p, w->alloc_stream);
    w->allocs.clear();
    if (!w->d_ur && !w->d_delta && !w->d_trace && !w->d_rows && !w->d_timers && !w->d_sched)
      return;
  }
  if (w->stream)
    cudaStreamSynchronize(w->stream);
  for (void* p : w->allocs)
    cudaFree(p);
  w->allocs.clear();
  cudaFree(w->d_ur);
  cudaFree(w->d_delta);
  cudaFree(w->d_trace);
  cudaFree(w->d_rows);
  cudaFree(w->d_timers);
  cudaFree(w->d_sched);
  if (w->own_stream && w->stream)
    cudaStreamDestroy(w->stream);
}

int qmc_walkers_create(qmc_system* s, int n_walkers, int delay_rank, qmc_walkers** out)
{
  if (!s || !out || n_walkers < 1 || delay_rank < 1 || delay_rank > 64 || delay_rank > s->h.norb)
    return fail(QMC_ERR_ARG, "bad walker batch arguments (1 <= delay_rank <= min(64, n_orb))");
  *out = nullptr;
  auto* w = new qmc_walkers_s;
  w->sys  = s;
  w->fp32 = s->fp32;
  int st  = alloc_walkers(w, s, n_walkers, delay_rank);
  if (st)
  {
    free_walkers(w);
    delete w;
    return st;
  }
  const int vw   = w->fp32 ? 4 : 2;
  const int nvec = s->h.npad / vw;
  w->threads     = std::min(256, std::max(std::max(64, 2 * delay_rank), round_up(nvec, 32)));
  w->tc_capable  = w->fp32 && w->threads >= 128 && delay_rank <= TC_KD && (s->h.comp & QMC_WF_DET);
  if (w->tc_capable)
  {
    if (dalloc(w->allocs, w->bytes, &w->dw.tci, (size_t)n_walkers * tc_image_floats(w->dw.npad, delay_rank)))
    {
      free_walkers(w);
      delete w;
      return QMC_ERR_OOM;
    }
    w->use_tc = true;
  }
  cudaError_t e  = cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess)
  {
    free_walkers(w);
    delete w;
    return fail(QMC_ERR_CUDA, cudaGetErrorString(e));
  }
  w->own_stream = true;
  *out          = w;
  return QMC_OK;
}
} // extern "C"

// a request-loop job's batch: memory stream-ordered from `pool` on `st`
// (which becomes the batch's stream); nothing here waits for the device
int walkers_create_pooled(qmc_system* s, int n_walkers, int delay_rank, cudaStream_t st, cudaMemPool_t pool,
                          qmc_walkers** out)
{
  if (!s || !out || n_walkers < 1 || delay_rank < 1 || delay_rank > 64 || delay_rank > s->h.norb || !st || !pool)
    return fail(QMC_ERR_ARG, "bad walker batch arguments");
  *out = nullptr;
  AllocScope scope(st, pool);
  auto* w         = new qmc_walkers_s;
  w->sys          = s;
  w->fp32         = s->fp32;
  w->stream       = st;
  w->own_stream   = false;
  w->alloc_stream = st;
  w->alloc_pool   = pool;
  int rc          = alloc_walkers(w, s, n_walkers, delay_rank);
  const int vw    = w->fp32 ? 4 : 2;
  w->threads      = std::min(256, std::max(std::max(64, 2 * delay_rank), round_up(s->h.npad / vw, 32)));
  w->tc_capable   = w->fp32 && w->threads >= 128 && delay_rank <= TC_KD && (s->h.comp & QMC_WF_DET);
  if (!rc && w->tc_capable)
  {
    rc        = dalloc(w->allocs, w->bytes, &w->dw.tci, (size_t)n_walkers * tc_image_floats(w->dw.npad, delay_rank));
    w->use_tc = rc == QMC_OK;
  }
  if (rc)
  {
    free_walkers(w);
    delete w;
    return rc;
  }
  *out = w;
  return QMC_OK;
}

extern "C" {

int qmc_walkers_destroy(qmc_walkers* w)
{
  if (!w)
    return QMC_OK;
  free_walkers(w);
  delete w;
  return QMC_OK;
}
int qmc_walkers_bytes(const qmc_walkers* w, size_t* bytes)
{
  if (!w || !bytes)
    return fail(QMC_ERR_ARG, "null pointer");
  *bytes = w->bytes;
  return QMC_OK;
}
int qmc_walkers_set_stream(qmc_walkers* w, void* stream)
{
  if (!w)
    return fail(QMC_ERR_ARG, "null pointer");
  cudaStreamSynchronize(w->stream);
  if (w->own_stream)
    cudaStreamDestroy(w->stream);
  w->own_stream = false;
  w->stream     = (cudaStream_t)stream;
  if (!stream)
  {
    cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking);
    w->own_stream = true;
  }
  return QMC_OK;
}
int qmc_walkers_launch_count(const qmc_walkers* w, int64_t* count)
{
  if (!w || !count)
    return fail(QMC_ERR_ARG, "null pointer");
  *count = w->launches;
  return QMC_OK;
}
int qmc_walkers_set_prefetch(qmc_walkers* w, int mode)
{
  if (!w || mode < QMC_PREFETCH_AUTO || mode > QMC_PREFETCH_ON)
    return fail(QMC_ERR_ARG, "bad prefetch mode");
  w->prefetch_mode = mode;
  return QMC_OK;
}

int qmc_walkers_set_schedule(qmc_walkers* w, int mode, int unit_moves, int ctas)
{
  if (!w || mode < QMC_SCHED_AUTO || mode > QMC_SCHED_QUEUE || unit_moves < 0 || ctas < 0)
    return fail(QMC_ERR_ARG, "bad schedule");
  w->sched_mode = mode;
  w->sched_unit = unit_moves ? unit_moves : QMC_SCHED_UNIT_DEFAULT;
  w->sched_ctas = ctas;
  return QMC_OK;
}

int qmc_walkers_set_threads(qmc_walkers* w, int threads)
{
  if (!w)
    return fail(QMC_ERR_ARG, "null handle");
  const int k = w->dw.k;
  if (threads % 32 || threads < std::max(64, 2 * k) || threads > 256)
    return fail(QMC_ERR_ARG, "threads per walker must be a multiple of 32 in [max(64, 2 delay), 256]");
  if (w->use_tc && threads < 128)
    return fail(QMC_ERR_ARG, "the tensor-core flush needs >= 128 threads per walker; switch it off first");
  w->threads = threads;
  return QMC_OK;
}
int qmc_walkers_get_config(const qmc_walkers* w, int* threads, int* delay, int* tensor_cores)
{
  if (!w)
    return fail(QMC_ERR_ARG, "null handle");
  if (threads)
    *threads = w->threads;
  if (delay)
    *delay = w->dw.k;
  if (tensor_cores)
    *tensor_cores = w->use_tc ? 1 : 0;
  return QMC_OK;
}
static int sweep_queue_ctas(const qmc_walkers* w);
static int sweep_queue_ctas_query(const qmc_walkers* w);
int qmc_walkers_occupancy(const qmc_walkers* w, int* walkers_per_sm)
{
  if (!w || !walkers_per_sm)
    return fail(QMC_ERR_ARG, "null pointer");
  const int q = sweep_queue_ctas(w);
  const int n = q < 0 ? -1
                      : sweep_occupancy(w->fp32, w->threads, w->dw.k, w->use_tc, (w->sys->h.comp & QMC_WF_J3) != 0,
                                        w->max_moves > 1, q > 0);
  if (n < 0)
    return fail(QMC_ERR_CUDA, "occupancy query failed");
  *walkers_per_sm = n;
  return QMC_OK;
}
int qmc_walkers_set_tensor_cores(qmc_walkers* w, int enable)
{
  if (!w)
    return fail(QMC_ERR_ARG, "null handle");
  if (enable && (!w->tc_capable || w->threads < 128))
    return fail(QMC_ERR_ARG, "tensor-core flush needs FP32 walkers, the determinant, delay rank <= 64 and >= 128 "
                             "threads per walker (480 or more orbitals per spin in FP32 give that)");
  w->use_tc = enable != 0;
  return QMC_OK;
}
int qmc_walkers_set_move_batching(qmc_walkers* w, int max_moves)
{
  if (!w || max_moves < 1 || max_moves > EPOCH_MAX)
    return fail(QMC_ERR_ARG, "null handle or max_moves outside [1, 4]");
  w->max_moves = max_moves;
  return QMC_OK;
}
int qmc_walkers_set_wait_limit(qmc_walkers* w, long long cycles)
{
  if (!w || cycles < 0)
    return fail(QMC_ERR_ARG, "null handle or negative wait limit");
  cudaError_t e = cudaStreamSynchronize(w->stream); // no launch in flight reads the old value
  if (e != cudaSuccess)
    return fail(QMC_ERR_CUDA, cudaGetErrorString(e));
  w->dw.wait_cycles = cycles;
  return QMC_OK;
}
int qmc_walkers_enable_timers(qmc_walkers* w, int enable)
{
  if (!w)
    return fail(QMC_ERR_ARG, "null handle");
  cudaStreamSynchronize(w->stream);
  cudaFree(w->d_timers);
  w->d_timers = nullptr;
  if (enable)
  {
    CK(cudaMalloc(&w->d_timers, (size_t)w->dw.W * NPHASE * sizeof(long long)));
    CK(cudaMemset(w->d_timers, 0, (size_t)w->dw.W * NPHASE * sizeof(long long)));
  }
  return QMC_OK;
}
int qmc_walkers_phase_times(qmc_walkers* w, double* ms, int* n_phases)
{
  if (!w || !ms)
    return fail(QMC_ERR_ARG, "null pointer");
  if (n_phases)
    *n_phases = NPHASE;
  if (!w->d_timers)
    return fail(QMC_ERR_STATE, "timers not enabled");
  std::vector<long long> t((size_t)w->dw.W * NPHASE);
  CK(cudaStreamSynchronize(w->stream));
  CK(cudaMemcpy(t.data(), w->d_timers, t.size() * sizeof(long long), cudaMemcpyDeviceToHost));
  int dev = 0, khz = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, dev);
  for (int p = 0; p < NPHASE; ++p)
  {
    double s = 0;
    for (int i = 0; i < w->dw.W; ++i)
      s += (double)t[(size_t)i * NPHASE + p];
    ms[p] = s / w->dw.W / (double)khz;
  }
  return QMC_OK;
}

int qmc_walkers_sync(qmc_walkers* w)
{
  if (!w)
    return fail(QMC_ERR_ARG, "null pointer");
  CK(cudaStreamSynchronize(w->stream));
  return device_status(w);
}

static int sync_rs(qmc_walkers* w)
{
  CK(launch_sync_rs(w->fp32, w->dw, w->stream));
  w->launches++;
  return QMC_OK;
}

int qmc_walkers_init_random(qmc_walkers* w, const uint32_t* seeds) { return walkers_init_random(w, seeds, true); }
} // extern "C"

// build_els on every walker's stream (host mt19937, then copied); sync =
// false leaves the copies and the SoA kernel in flight (the sources are
// pageable, so they are staged before each call returns)
int walkers_init_random(qmc_walkers* w, const uint32_t* seeds, bool sync)
{
  if (!w || !seeds)
    return fail(QMC_ERR_ARG, "null pointer");
  const int W = w->dw.W, N = w->dw.N;
  std::vector<double> R((size_t)W * N * 3);
  std::vector<uint32_t> mt((size_t)W * (MT_N + 1));
  for (int i = 0; i < W; ++i)
  {
    MTState st;
    mt_seed_host(st, seeds[i]);
    for (int e = 0; e < N; ++e)
    {
      double u[3];
      for (int c = 0; c < 3; ++c)
      {
        const uint32_t w0 = mt_next_host(st);
        const uint32_t w1 = mt_next_host(st);
        u[c]              = canonical_double(w0, w1);
      }
      qmc_host::to_cart(w->sys->h.lattice, u, &R[((size_t)i * N + e) * 3]);
    }
    std::memcpy(&mt[(size_t)i * (MT_N + 1)], st.mt, sizeof(st.mt));
    mt[(size_t)i * (MT_N + 1) + MT_N] = (uint32_t)st.mti;
  }
  CK(cudaMemcpyAsync(w->dw.R, R.data(), R.size() * sizeof(double), cudaMemcpyHostToDevice, w->stream));
  CK(cudaMemcpyAsync(w->dw.mt, mt.data(), mt.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, w->stream));
  int st = sync_rs(w);
  if (st)
    return st;
  if (sync)
    CK(cudaStreamSynchronize(w->stream));
  return QMC_OK;
}

extern "C" {
int qmc_walkers_set_positions(qmc_walkers* w, const double* R)
{
  if (!w || !R)
    return fail(QMC_ERR_ARG, "null pointer");
  CK(cudaMemcpyAsync(w->dw.R, R, (size_t)w->dw.W * w->dw.N * 3 * sizeof(double), cudaMemcpyHostToDevice, w->stream));
  int st = sync_rs(w);
  if (st)
    return st;
  CK(cudaStreamSynchronize(w->stream));
  return QMC_OK;
}
int qmc_walkers_get_positions(qmc_walkers* w, double* R)
{
  if (!w || !R)
    return fail(QMC_ERR_ARG, "null pointer");
  CK(cudaMemcpyAsync(R, w->dw.R, (size_t)w->dw.W * w->dw.N * 3 * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaStreamSynchronize(w->stream));
  return QMC_OK;
}

// ------------------------------------------------------------ verbs -----
static int verb(qmc_walkers* w, VerbArgs a)
{
  CK(launch_verb(w->fp32, w->sys->d, w->dw, a, w->threads, w->dw.k, w->stream));
  w->launches++;
  return QMC_OK;
}
static int check_iat(qmc_walkers* w, int iat)
{
  if (!w)
    return fail(QMC_ERR_ARG, "null handle");
  if (iat < 0 || iat >= w->dw.N)
    return fail(QMC_ERR_ARG, "electron index out of range");
  return QMC_OK;
}

int qmc_pset_update(qmc_walkers* w) { return w ? QMC_OK : fail(QMC_ERR_ARG, "null handle"); }
int qmc_pset_done(qmc_walkers* w) { return w ? QMC_OK : fail(QMC_ERR_ARG, "null handle"); }
int qmc_pset_set_active(qmc_walkers* w, int iat) { return check_iat(w, iat); }

int qmc_pset_make_move(qmc_walkers* w, int iat, const double* displ)
{
  int st = check_iat(w, iat);
  if (st)
    return st;
  if (!displ)
    return fail(QMC_ERR_ARG, "null displacement");
  CK(cudaMemcpyAsync(w->d_displ, displ, 3 * w->dw.W * sizeof(double), cudaMemcpyHostToDevice, w->stream));
  VerbArgs a{};
  a.op    = VERB_MAKE_MOVE;
  a.iat   = iat;
  a.displ = w->d_displ;
  return verb(w, a);
}
static int flags_verb(qmc_walkers* w, int op, int iat, const int* accept)
{
  int st = check_iat(w, iat);
  if (st)
    return st;
  if (!accept)
    return fail(QMC_ERR_ARG, "null accept flags");
  CK(cudaMemcpyAsync(w->d_flags, accept, w->dw.W * sizeof(int), cudaMemcpyHostToDevice, w->stream));
  VerbArgs a{};
  a.op    = op;
  a.iat   = iat;
  a.flags = w->d_flags;
  if ((st = verb(w, a)))
    return st;
  CK(cudaStreamSynchronize(w->stream));
  return device_status(w);
}
int qmc_pset_accept_reject(qmc_walkers* w, int iat, const int* accept)
{
  return flags_verb(w, VERB_PSET_ACCEPT, iat, accept);
}
int qmc_wf_accept_restore(qmc_walkers* w, int iat, const int* accept)
{
  return flags_verb(w, VERB_WF_ACCEPT, iat, accept);
}

int qmc_pset_get_temp_rows(qmc_walkers* w, double* aa_r, double* aa_dr, double* ab_r, double* ab_dr)
{
  if (!w)
    return fail(QMC_ERR_ARG, "null handle");
  const size_t W = w->dw.W, N = w->dw.N, I = w->dw.I;
  const size_t need = W * (4 * N + 4 * I);
  if (w->cap_rows < need)
  {
    cudaFree(w->d_rows);
    CK(cudaMalloc(&w->d_rows, need * sizeof(double)));
    w->cap_rows = need;
  }
  VerbArgs a{};
  a.op    = VERB_TEMP_ROWS;
  a.iat   = 0;
  a.aa_r  = w->d_rows;
  a.aa_dr = a.aa_r + W * N;
  a.ab_r  = a.aa_dr + W * N * 3;
  a.ab_dr = a.ab_r + W * I;
  int st  = verb(w, a);
  if (st)
    return st;
  if (aa_r)
    CK(cudaMemcpyAsync(aa_r, a.aa_r, W * N * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  if (aa_dr)
    CK(cudaMemcpyAsync(aa_dr, a.aa_dr, W * N * 3 * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  if (ab_r)
    CK(cudaMemcpyAsync(ab_r, a.ab_r, W * I * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  if (ab_dr)
    CK(cudaMemcpyAsync(ab_dr, a.ab_dr, W * I * 3 * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaStreamSynchronize(w->stream));
  return QMC_OK;
}

static int ensure_lu(qmc_walkers* w)
{
  if (w->dw.lu)
    return QMC_OK;
  AllocScope scope(w->alloc_stream, w->alloc_pool);
  return dalloc(w->allocs, w->bytes, &w->dw.lu, (size_t)w->dw.W * 2 * w->dw.n * w->dw.npad);
}

// FP64 refresh of both inverses from the current positions
} // extern "C"

int recompute_dets(qmc_walkers* w)
{
  int st = ensure_lu(w);
  if (st)
    return st;
  CK(launch_spo_matrix(w->fp32, w->sys->d, w->dw, true, w->stream));
  CK(launch_gj_inverse(w->fp32, w->sys->d, w->dw, 512, 2, w->stream));
  w->launches += 2;
  return QMC_OK;
}

extern "C" {

int qmc_wf_evaluate_log(qmc_walkers* w, double* logpsi)
{
  int st = evaluate_log_launch(w);
  if (st)
    return st;
  if (logpsi)
    CK(cudaMemcpyAsync(logpsi, w->dw.logpsi, w->dw.W * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaStreamSynchronize(w->stream));
  return device_status(w);
}
} // extern "C"

// evaluateLog's launches on the batch's stream, without waiting for them
// (errors land in the batch's status word)
int evaluate_log_launch(qmc_walkers* w)
{
  if (!w)
    return fail(QMC_ERR_ARG, "null handle");
  const int comp = w->sys->h.comp;
  int st         = 0;
  if (comp & QMC_WF_DET)
    if ((st = recompute_dets(w)))
      return st;
  if (comp & (QMC_WF_J1 | QMC_WF_J2))
  {
    CK(launch_jastrow_recompute(w->fp32, w->sys->d, w->dw, 256, w->stream));
    w->launches++;
  }
  if (comp & QMC_WF_J3)
  {
    CK(launch_j3_recompute(w->fp32, w->sys->d, w->dw, 256, w->stream));
    w->launches++;
  }
  CK(launch_gl(w->fp32, w->sys->d, w->dw, w->threads, w->stream));
  w->launches++;
  w->ratio_moves = false;
  std::vector<MoveState> ms(w->dw.W);
  for (auto& m : ms)
  {
    std::memset(&m, 0, sizeof(m));
    m.active       = -1;
    m.invrow_id[0] = m.invrow_id[1] = -1;
    m.partial[0] = m.partial[1] = 1;
    m.j_partial                 = 1;
  }
  CK(cudaMemcpyAsync(w->dw.ms, ms.data(), ms.size() * sizeof(MoveState), cudaMemcpyHostToDevice, w->stream));
  return QMC_OK;
}

extern "C" {

int qmc_wf_eval_grad(qmc_walkers* w, int iat, double* grad)
{
  int st = check_iat(w, iat);
  if (st)
    return st;
  VerbArgs a{};
  a.op  = VERB_EVAL_GRAD;
  a.iat = iat;
  if ((st = verb(w, a)))
    return st;
  if (grad)
    CK(cudaMemcpyAsync(grad, w->dw.out_grad, 3 * w->dw.W * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaStreamSynchronize(w->stream));
  return device_status(w);
}
static int ratio_verb(qmc_walkers* w, int op, int iat, double* ratio, double* grad)
{
  int st = check_iat(w, iat);
  if (st)
    return st;
  VerbArgs a{};
  a.op  = op;
  a.iat = iat;
  if ((st = verb(w, a)))
    return st;
  if (ratio)
    CK(cudaMemcpyAsync(ratio, w->dw.out_ratio, w->dw.W * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  if (grad)
    CK(cudaMemcpyAsync(grad, w->dw.out_grad, 3 * w->dw.W * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaStreamSynchronize(w->stream));
  return device_status(w);
}
int qmc_wf_ratio_grad(qmc_walkers* w, int iat, double* ratio, double* grad)
{
  return ratio_verb(w, VERB_RATIO_GRAD, iat, ratio, grad);
}
int qmc_wf_ratio(qmc_walkers* w, int iat, double* ratio)
{
  if (w)
    w->ratio_moves = true;
  return ratio_verb(w, VERB_RATIO, iat, ratio, nullptr);
}

int qmc_spo_evaluate_batch(qmc_walkers* w, int iat, double* v_dev, double* g_dev, double* h_dev)
{
  int st = check_iat(w, iat);
  if (st)
    return st;
  if (!v_dev && !g_dev && !h_dev)
    return fail(QMC_ERR_ARG, "no output buffer");
  // the positions go through the qmc_step scratch ([W][4] doubles, >= [W][3])
  CK(launch_active_pos(w->dw, iat, w->d_step, w->stream));
  CK(launch_spo_points(w->fp32, w->sys->d, w->dw.W, w->d_step, v_dev, g_dev, h_dev, !g_dev && !h_dev, w->stream));
  w->launches += 2;
  return QMC_OK;
}

int qmc_step(qmc_walkers* w, int iat, double accept, const double* ur, const double* delta, int* accepted)
{
  int st = check_iat(w, iat);
  if (st)
    return st;
  if (!ur || !delta)
    return fail(QMC_ERR_ARG, "null ur or delta");
  const size_t W = w->dw.W;
  std::vector<double> in(4 * W);
  for (size_t i = 0; i < W; ++i)
  {
    in[4 * i] = ur[i];
    for (int c = 0; c < 3; ++c)
      in[4 * i + 1 + c] = delta[3 * i + c];
  }
  CK(cudaMemcpyAsync(w->d_step, in.data(), 4 * W * sizeof(double), cudaMemcpyHostToDevice, w->stream));
  CK(launch_step(w->fp32, (w->sys->h.comp & QMC_WF_J3) != 0, w->sys->d, w->dw, iat, accept, w->d_step, w->d_flags,
                 w->threads, w->stream));
  w->launches++;
  if (accepted)
    CK(cudaMemcpyAsync(accepted, w->d_flags, W * sizeof(int), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaStreamSynchronize(w->stream));
  return device_status(w);
}

int qmc_wf_complete_updates(qmc_walkers* w)
{
  if (!w)
    return fail(QMC_ERR_ARG, "null handle");
  VerbArgs a{};
  a.op   = VERB_COMPLETE;
  int st = verb(w, a);
  if (st)
    return st;
  CK(cudaStreamSynchronize(w->stream));
  return device_status(w);
}

int qmc_wf_evaluate_gl(qmc_walkers* w, double* G, double* L, double* logpsi)
{
  if (!w)
    return fail(QMC_ERR_ARG, "null handle");
  if (w->ratio_moves && (w->sys->h.comp & QMC_WF_DET))
  {
    // derivative rows of the determinants left in ratio-only mode
    CK(launch_spo_matrix(w->fp32, w->sys->d, w->dw, false, w->stream, true));
    w->launches++;
  }
  CK(launch_gl(w->fp32, w->sys->d, w->dw, w->threads, w->stream));
  w->launches++;
  const size_t W = w->dw.W, N = w->dw.N;
  if (G)
    CK(cudaMemcpyAsync(G, w->dw.G, W * N * 3 * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  if (L)
    CK(cudaMemcpyAsync(L, w->dw.L, W * N * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  if (logpsi)
    CK(cudaMemcpyAsync(logpsi, w->dw.logpsi, W * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaStreamSynchronize(w->stream));
  return QMC_OK;
}

int qmc_wf_components(qmc_walkers* w, double* comp)
{
  if (!w || !comp)
    return fail(QMC_ERR_ARG, "null pointer");
  const size_t W = w->dw.W;
  std::vector<double> dl(2 * W), dp(2 * W), jl(3 * W);
  CK(cudaMemcpyAsync(dl.data(), w->dw.det_log, 2 * W * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(dp.data(), w->dw.det_phase, 2 * W * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(jl.data(), w->dw.j_log, 3 * W * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaStreamSynchronize(w->stream));
  for (size_t i = 0; i < W; ++i)
  {
    comp[7 * i + 0] = dl[2 * i];
    comp[7 * i + 1] = dl[2 * i + 1];
    comp[7 * i + 2] = dp[2 * i];
    comp[7 * i + 3] = dp[2 * i + 1];
    comp[7 * i + 4] = jl[3 * i];
    comp[7 * i + 5] = jl[3 * i + 1];
    comp[7 * i + 6] = jl[3 * i + 2];
  }
  return QMC_OK;
}

// Ainv with the pending delayed rows applied: Ainv - (Ainv U^T - E)(Binv V),
// evaluated on a host copy (an inspection accessor, not on the move path).
int qmc_wf_get_inverse(qmc_walkers* w, int walker, int spin, double* psiM)
{
  if (!w || !psiM || walker < 0 || walker >= w->dw.W || spin < 0 || spin > 1)
    return fail(QMC_ERR_ARG, "bad arguments");
  const size_t n = w->dw.n, np = w->dw.npad, k = w->dw.k, es = w->fp32 ? 4 : 8;
  std::vector<unsigned char> a(n * np * es), u(k * np * es), v(k * np * es);
  std::vector<double> B(k * k);
  std::vector<int> dl(k);
  int dc = 0;
  const size_t mat = ((size_t)walker * 2 + spin);
  CK(cudaMemcpy(a.data(), (unsigned char*)w->dw.Ainv + mat * n * np * es, a.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(u.data(), (unsigned char*)w->dw.U + mat * k * np * es, u.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(v.data(), (unsigned char*)w->dw.V + mat * k * np * es, v.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(B.data(), w->dw.Binv + mat * k * k, B.size() * sizeof(double), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(dl.data(), w->dw.delay_list + mat * k, k * sizeof(int), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&dc, w->dw.delay_count + mat, sizeof(int), cudaMemcpyDeviceToHost));
  auto at = [&](const std::vector<unsigned char>& buf, size_t i) -> double {
    return es == 4 ? (double)((const float*)buf.data())[i] : ((const double*)buf.data())[i];
  };
  std::vector<double> A(n * n);
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j < n; ++j)
      A[i * n + j] = at(a, i * np + j);
  if (dc > 0)
  {
    std::vector<double> tm(n * dc), U2(dc * n, 0.0);
    for (size_t i = 0; i < n; ++i)
      for (int d = 0; d < dc; ++d)
      {
        double s = 0;
        for (size_t j = 0; j < n; ++j)
          s += at(u, d * np + j) * A[i * n + j];
        tm[i * dc + d] = s - (dl[d] == (int)i ? 1.0 : 0.0);
      }
    for (int b = 0; b < dc; ++b)
      for (int aa = 0; aa < dc; ++aa)
        for (size_t j = 0; j < n; ++j)
          U2[b * n + j] += B[b * k + aa] * at(v, aa * np + j);
    for (size_t i = 0; i < n; ++i)
      for (int d = 0; d < dc; ++d)
        for (size_t j = 0; j < n; ++j)
          A[i * n + j] -= tm[i * dc + d] * U2[d * n + j];
  }
  std::memcpy(psiM, A.data(), A.size() * sizeof(double));
  return QMC_OK;
}

// ------------------------------------------------------------ sweep -----
// CTAs of a work-queue sweep launch for this batch, 0 for the static form
// (one CTA per walker), -1 if the occupancy query failed.  AUTO is the
// queue, with every resident CTA slot (walkers per SM x SMs) taking units:
// the slots beyond the walkers are the CTAs that wait for a walker, so no
// walker waits for a CTA, and where the walkers outnumber the slots they
// take turns on them.
static int sweep_queue_ctas(const qmc_walkers* w)
{
  if (w->sched_mode == QMC_SCHED_STATIC)
    return 0;
  // the answer for the present settings, kept from the last call
  const int key[6] = {w->sched_mode, w->sched_ctas, w->threads, (int)w->use_tc, w->max_moves, 1};
  if (std::equal(key, key + 6, w->sched_key))
    return w->sched_cached;
  const int n = sweep_queue_ctas_query(w);
  if (n >= 0)
  {
    std::copy(key, key + 6, w->sched_key);
    w->sched_cached = n;
  }
  return n;
}

static int sweep_queue_ctas_query(const qmc_walkers* w)
{
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))
    return -1;
  if (w->sched_ctas > 0)
    return w->sched_ctas;
  const int per_sm = sweep_occupancy(w->fp32, w->threads, w->dw.k, w->use_tc, (w->sys->h.comp & QMC_WF_J3) != 0,
                                     w->max_moves > 1, true);
  if (per_sm < 1)
    return -1;
  return per_sm * sms;
}

static int sweep_steps(qmc_walkers* w, int n_steps, int n_substeps, double accept, int rng_mode, const double* ur,
                       const double* delta, int recompute_every, double* trace, bool async)
{
  const size_t W = w->dw.W, N = w->dw.N;
  if (rng_mode == QMC_RNG_HOST)
  {
    const size_t need = W * n_substeps * N;
    if (w->cap_rng < need)
    {
      cudaFree(w->d_ur);
      cudaFree(w->d_delta);
      CK(cudaMalloc(&w->d_ur, need * sizeof(double)));
      CK(cudaMalloc(&w->d_delta, 3 * need * sizeof(double)));
      w->cap_rng = need;
    }
  }
  if (trace)
  {
    const size_t need = W * n_substeps * N * 8;
    if (w->cap_trace < need)
    {
      cudaFree(w->d_trace);
      CK(cudaMalloc(&w->d_trace, need * sizeof(double)));
      w->cap_trace = need;
    }
  }
  SweepTask task = sweep_task(w, 0);
  task.rng_mode  = rng_mode;
  task.ur        = w->d_ur;
  task.delta     = w->d_delta;
  task.trace     = trace ? w->d_trace : nullptr;
  CK(cudaMemcpyAsync(w->d_task, &task, sizeof(task), cudaMemcpyHostToDevice, w->stream));
  const int queue_ctas = sweep_queue_ctas(w);
  if (queue_ctas < 0)
    return fail(QMC_ERR_CUDA, "occupancy query failed");
  const size_t total_units = W * (size_t)sweep_queue_units((int)N, w->sys->h.n_up, n_substeps, w->sched_unit);
  const size_t n_sched     = queue_ctas ? sweep_queue_words((int)W, queue_ctas, total_units) : 0;
  if (n_sched > (size_t)INT32_MAX)
    return fail(QMC_ERR_ARG, "too many work-queue units in one launch: take longer units");
  if (w->cap_sched < n_sched)
  {
    cudaFree(w->d_sched);
    w->d_sched = nullptr;
    CK(cudaMalloc(&w->d_sched, n_sched * sizeof(int)));
    w->cap_sched = n_sched;
  }
  for (int step = 0; step < n_steps; ++step)
  {
    if (rng_mode == QMC_RNG_HOST)
    {
      const size_t blk = W * n_substeps * N;
      CK(cudaMemcpyAsync(w->d_ur, ur + step * blk, blk * sizeof(double), cudaMemcpyHostToDevice, w->stream));
      CK(cudaMemcpyAsync(w->d_delta, delta + step * blk * 3, 3 * blk * sizeof(double), cudaMemcpyHostToDevice,
                         w->stream));
    }
    const bool j3 = (w->sys->h.comp & QMC_WF_J3) != 0;
    if (queue_ctas > 0)
    {
      CK(cudaMemsetAsync(w->d_sched, 0, n_sched * sizeof(int), w->stream));
      const QueueLaunch q{w->d_task,    1,          (int)W, (int)total_units, n_substeps, w->sched_unit,
                          queue_ctas, w->threads, accept, w->use_tc,      w->d_sched};
      CK(launch_sweep_queue(w->fp32, q, w->dw.k, j3, w->max_moves > 1, w->stream));
    }
    else
      CK(launch_sweep(w->fp32, w->d_task, 1, (int)W, n_substeps, accept, w->threads, w->dw.npad, w->dw.k,
                      w->stream, w->use_tc, j3, w->max_moves > 1));
    w->launches++;
    if (trace)
      CK(cudaMemcpyAsync(trace + (size_t)step * W * n_substeps * N * 8, w->d_trace,
                         W * n_substeps * N * 8 * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
    ++w->steps_done;
    if (recompute_every > 0 && w->steps_done % recompute_every == 0 && (w->sys->h.comp & QMC_WF_DET))
    {
      int st = recompute_dets(w);
      if (st)
        return st;
      CK(launch_gl(w->fp32, w->sys->d, w->dw, w->threads, w->stream));
      w->launches++;
    }
  }
  if (!async)
  {
    CK(cudaStreamSynchronize(w->stream));
    return device_status(w);
  }
  return QMC_OK;
}

} // extern "C"

SweepTask sweep_task(qmc_walkers* w, int first_block)
{
  SweepTask task{};
  task.sys         = w->sys->d;
  task.dw          = w->dw;
  task.rng_mode    = QMC_RNG_DEVICE;
  task.first_block = first_block;
  task.timers      = w->d_timers;
  task.tc          = w->use_tc ? 1 : 0;
  task.max_moves   = w->max_moves;
  // next-move L2 prefetch only while the batch's in-flight stencils (16 rows
  // of 4 npad coefficients per walker) stay well inside the 126 MB L2
  task.prefetch = w->prefetch_mode == QMC_PREFETCH_ON ||
      (w->prefetch_mode == QMC_PREFETCH_AUTO && (double)w->dw.W * 16 * 4 * w->dw.npad * (w->fp32 ? 4 : 8) <= 32.0e6);
  return task;
}

extern "C" {

int qmc_sweep(qmc_walkers* w, const qmc_sweep_opts* o)
{
  if (!w || !o || o->n_steps < 0 || o->n_substeps < 1)
    return fail(QMC_ERR_ARG, "bad sweep options");
  if (o->rng_mode == QMC_RNG_HOST && (!o->ur || !o->delta))
    return fail(QMC_ERR_ARG, "QMC_RNG_HOST needs ur and delta");
  CK(cudaMemsetAsync(w->dw.accepted, 0, w->dw.W * sizeof(long long), w->stream));
  int st = sweep_steps(w, o->n_steps, o->n_substeps, o->accept, o->rng_mode, o->ur, o->delta, o->recompute_every,
                       o->trace, false);
  if (st)
    return st;
  if (o->n_accepted)
    CK(cudaMemcpy(o->n_accepted, w->dw.accepted, w->dw.W * sizeof(long long), cudaMemcpyDeviceToHost));
  if (o->logpsi)
    CK(cudaMemcpy(o->logpsi, w->dw.logpsi, w->dw.W * sizeof(double), cudaMemcpyDeviceToHost));
  return QMC_OK;
}

int qmc_sweep_async(qmc_walkers* w, int n_steps, int n_substeps, double accept, int recompute_every)
{
  if (!w || n_steps < 0 || n_substeps < 1)
    return fail(QMC_ERR_ARG, "bad sweep options");
  return sweep_steps(w, n_steps, n_substeps, accept, QMC_RNG_DEVICE, nullptr, nullptr, recompute_every, nullptr,
                     true);
}

int qmc_sweep_results(qmc_walkers* w, int64_t* n_accepted, double* logpsi)
{
  if (!w)
    return fail(QMC_ERR_ARG, "null handle");
  if (n_accepted)
    CK(cudaMemcpyAsync(n_accepted, w->dw.accepted, w->dw.W * sizeof(long long), cudaMemcpyDeviceToHost, w->stream));
  if (logpsi)
    CK(cudaMemcpyAsync(logpsi, w->dw.logpsi, w->dw.W * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaStreamSynchronize(w->stream));
  return device_status(w);
}

// ------------------------------------------------- DelayedUpdate engine --
struct qmc_detengine_s
{
  qmc_walkers_s w;
};

static void to_dev_elems(const qmc_walkers_s* w, const double* src, size_t n, std::vector<unsigned char>& buf)
{
  const size_t es = w->fp32 ? 4 : 8;
  buf.assign(n * es, 0);
  for (size_t i = 0; i < n; ++i)
    if (w->fp32)
      reinterpret_cast<float*>(buf.data())[i] = (float)src[i];
    else
      reinterpret_cast<double*>(buf.data())[i] = src[i];
}
static double dev_elem(const qmc_walkers_s* w, const std::vector<unsigned char>& buf, size_t i)
{
  return w->fp32 ? (double)reinterpret_cast<const float*>(buf.data())[i] : reinterpret_cast<const double*>(buf.data())[i];
}

int qmc_detengine_create_prec(int n, int delay, int precision, qmc_detengine_s** out)
{
  if (!out || n < 1 || delay < 1 || delay > 64 || delay > n)
    return fail(QMC_ERR_ARG, "bad engine size");
  auto* e       = new qmc_detengine_s;
  auto* w       = &e->w;
  DevWalkers& d = w->dw;
  std::memset(&d, 0, sizeof(d));
  d.W = 1, d.N = n, d.Npad = round_up(n, 32), d.n = n, d.npad = round_up(n, 32), d.I = 0, d.k = delay;
  d.wait_cycles    = kTcWaitCycles;
  w->fp32          = precision == QMC_PREC_MIXED;
  const size_t es  = w->fp32 ? 4 : 8;
  const size_t np  = d.npad, K = delay;
  auto& L          = w->allocs;
  auto& B          = w->bytes;
  int st           = 0;
  auto Tm          = [&](void** p, size_t c) {
    unsigned char* q = nullptr;
    int r            = dalloc(L, B, &q, c * es);
    *p               = q;
    return r;
  };
  st |= Tm(&d.Ainv, 2 * n * np);
  st |= Tm(&d.dpsiM, 2 * 3 * n * np);
  st |= Tm(&d.d2psiM, 2 * n * np);
  st |= Tm(&d.U, 2 * K * np);
  st |= Tm(&d.V, 2 * K * np);
  st |= dalloc(L, B, &d.Binv, 2 * K * K);
  st |= dalloc(L, B, &d.delay_list, 2 * K);
  st |= dalloc(L, B, &d.delay_count, 2);
  st |= dalloc(L, B, &d.det_log, 2);
  st |= dalloc(L, B, &d.det_phase, 2);
  st |= Tm(&d.invRow, np);
  st |= Tm(&d.psiV, np);
  st |= Tm(&d.dpsiV, 3 * np);
  st |= Tm(&d.d2psiV, np);
  st |= Tm(&d.U2, K * np);
  st |= Tm(&d.tm, n * K);
  st |= dalloc(L, B, &d.lu, 2 * n * np);
  st |= dalloc(L, B, &d.status, 1);
  st |= dalloc(L, B, &d.ms, 1);
  w->tc_capable = w->fp32 && delay <= TC_KD;
  if (w->tc_capable)
  {
    st |= dalloc(L, B, &d.tci, tc_image_floats(d.npad, delay));
    w->use_tc = true;
  }
  if (st)
  {
    free_walkers(w);
    delete e;
    return QMC_ERR_OOM;
  }
  cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking);
  w->own_stream = true;
  *out          = e;
  return QMC_OK;
}
int qmc_detengine_create(int n, int delay, qmc_detengine_s** out)
{
  return qmc_detengine_create_prec(n, delay, QMC_PREC_FP64, out);
}
int qmc_detengine_set_tensor_cores(qmc_detengine_s* e, int enable)
{
  if (!e)
    return fail(QMC_ERR_ARG, "null handle");
  if (enable && !e->w.tc_capable)
    return fail(QMC_ERR_ARG, "tensor-core flush needs an FP32 engine with delay rank <= 64");
  e->w.use_tc = enable != 0;
  return QMC_OK;
}
int qmc_detengine_destroy(qmc_detengine_s* e)
{
  if (!e)
    return QMC_OK;
  free_walkers(&e->w);
  delete e;
  return QMC_OK;
}
int qmc_detengine_invert_transpose(qmc_detengine_s* e, const double* a, double* logdet, double* phase)
{
  if (!e || !a)
    return fail(QMC_ERR_ARG, "null pointer");
  auto* w        = &e->w;
  const size_t n = w->dw.n, np = w->dw.npad;
  std::vector<double> m(n * np, 0.0);
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j < n; ++j)
      m[i * np + j] = a[i * n + j];
  CK(cudaMemcpyAsync(w->dw.lu, m.data(), m.size() * sizeof(double), cudaMemcpyHostToDevice, w->stream));
  CK(launch_gj_inverse(w->fp32, nullptr, w->dw, 256, 1, w->stream));
  double lg = 0, ph = 0;
  CK(cudaMemcpyAsync(&lg, w->dw.det_log, sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(&ph, w->dw.det_phase, sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaStreamSynchronize(w->stream));
  if (logdet)
    *logdet = lg;
  if (phase)
    *phase = ph;
  return device_status(w);
}
int qmc_detengine_get_inv_row(qmc_detengine_s* e, int row, double* inv_row)
{
  if (!e || !inv_row || row < 0 || row >= e->w.dw.n)
    return fail(QMC_ERR_ARG, "bad arguments");
  auto* w = &e->w;
  CK(launch_det_engine(w->fp32, DETENG_GET_INV_ROW, w->dw, row, w->dw.k, w->stream, w->use_tc));
  std::vector<unsigned char> buf(w->dw.n * (w->fp32 ? 4 : 8));
  CK(cudaMemcpyAsync(buf.data(), w->dw.invRow, buf.size(), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaStreamSynchronize(w->stream));
  for (int i = 0; i < w->dw.n; ++i)
    inv_row[i] = dev_elem(w, buf, i);
  return device_status(w);
}
int qmc_detengine_accept_row(qmc_detengine_s* e, int row, const double* psiv)
{
  if (!e || !psiv || row < 0 || row >= e->w.dw.n)
    return fail(QMC_ERR_ARG, "bad arguments");
  auto* w = &e->w;
  std::vector<double> p(w->dw.npad, 0.0);
  std::memcpy(p.data(), psiv, w->dw.n * sizeof(double));
  std::vector<unsigned char> buf;
  to_dev_elems(w, p.data(), p.size(), buf);
  CK(cudaMemcpyAsync(w->dw.psiV, buf.data(), buf.size(), cudaMemcpyHostToDevice, w->stream));
  CK(launch_det_engine(w->fp32, DETENG_ACCEPT_ROW, w->dw, row, w->dw.k, w->stream, w->use_tc));
  CK(cudaStreamSynchronize(w->stream));
  return device_status(w);
}
int qmc_detengine_update_inv_mat(qmc_detengine_s* e)
{
  if (!e)
    return fail(QMC_ERR_ARG, "null pointer");
  auto* w = &e->w;
  CK(launch_det_engine(w->fp32, DETENG_UPDATE, w->dw, 0, w->dw.k, w->stream, w->use_tc));
  CK(cudaStreamSynchronize(w->stream));
  return device_status(w);
}
int qmc_detengine_get_ainv(qmc_detengine_s* e, double* ainv)
{
  if (!e || !ainv)
    return fail(QMC_ERR_ARG, "null pointer");
  auto* w        = &e->w;
  const size_t n = w->dw.n, np = w->dw.npad;
  std::vector<unsigned char> buf(n * np * (w->fp32 ? 4 : 8));
  CK(cudaMemcpy(buf.data(), w->dw.Ainv, buf.size(), cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j < n; ++j)
      ainv[i * n + j] = dev_elem(w, buf, i * np + j);
  return QMC_OK;
}

// ------------------------------------------- allocation-free inverse --
} // extern "C"

// Working storage of qmc_invert_transpose_noalloc: the FP64 working copy of
// the matrix (row stride n) followed by four words (log|det|, phase, the
// delay count the inverse kernel resets, the device error bits).  It lives
// in the library's static device memory, one copy per device, so the call
// needs no cudaMalloc; its size fixes the largest n.
static constexpr size_t kNoallocLU = (size_t)QMC_NOALLOC_MAX_N * QMC_NOALLOC_MAX_N;
static __device__ __align__(256) double g_noalloc_scratch[kNoallocLU + 4];

static std::mutex g_noalloc_mu;
static constexpr int kNoallocDevices = 64;
static void* g_noalloc_base[kNoallocDevices];

// Device address of the static scratch on the current device, looked up
// once per device (the set-up step: it may load the library's device code)
static int noalloc_scratch(double** out)
{
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoallocDevices)
    return fail(QMC_ERR_CUDA, "device ordinal beyond the scratch table");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_base[dev])
  {
    void* p = nullptr;
    CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_base[dev] = p;
  }
  *out = static_cast<double*>(g_noalloc_base[dev]);
  return QMC_OK;
}

extern "C" {

int qmc_invert_transpose_noalloc(int n, const double* a, double* psim, double* logdet, double* phase,
                                 void* stream)
{
  if (n < 1 || n > QMC_NOALLOC_MAX_N)
    return fail(QMC_ERR_ARG, "qmc_invert_transpose_noalloc: n = " + std::to_string(n) +
                                 " is outside 1.." + std::to_string(QMC_NOALLOC_MAX_N) +
                                 ", the size of the static scratch");
  if (!a || !psim)
    return fail(QMC_ERR_ARG, "qmc_invert_transpose_noalloc: null device pointer");
  double* base = nullptr;
  if (int r = noalloc_scratch(&base))
    return r;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* words   = base + kNoallocLU;
  unsigned* stat  = reinterpret_cast<unsigned*>(words + 3);
  // a one-walker, one-spin view whose matrices are the caller's buffers and
  // the static scratch (row stride n)
  DevWalkers v;
  std::memset(&v, 0, sizeof(v));
  v.W = 1, v.N = n, v.Npad = n, v.n = n, v.npad = n, v.k = 1;
  v.lu          = base;
  v.Ainv        = psim;
  v.det_log     = words;
  v.det_phase   = words + 1;
  v.delay_count = reinterpret_cast<int*>(words + 2);
  v.status      = stat;
  // the error bits are only ever OR-ed in by the kernel: clear them first
  CK(cudaMemsetAsync(stat, 0, sizeof(unsigned), st));
  CK(cudaMemcpyAsync(base, a, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  CK(launch_gj_inverse(false, nullptr, v, 256, 1, st));
  double hw[4];
  CK(cudaMemcpyAsync(hw, words, sizeof(hw), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (logdet)
    *logdet = hw[0];
  if (phase)
    *phase = hw[1];
  unsigned bits = 0;
  std::memcpy(&bits, &hw[3], sizeof(bits));
  if (bits & DEV_ERR_SINGULAR)
    return fail(QMC_ERR_SINGULAR, "zero pivot in the FP64 inverse");
  if (bits)
    return fail(QMC_ERR_CUDA, "device error bits set");
  return QMC_OK;
}

} // extern "C"
