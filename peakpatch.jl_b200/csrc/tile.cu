// tile.cu — run_tile on one GPU (src/Pipeline.jl:66-325).
//
// Phase 0 (host): cosmology tables, fcrit = fsc_of_z(z_out), filter bank
//   sorted by Rf descending, nhunt = min(nbuff-1, floor(1.75 Rfmax/alatt)).
// Phase 1: Threefry noise -> R2C -> sqrt(P) -> C2R = delta; delta_k = R2C(delta);
//   1LPT (3 C2R), 2LPT (6 C2R, src2, R2C, 3 C2R), Laplacian (ioutshear >= 1).
// Phase 2: per filter (largest first): window -> C2R -> peak finder with a
//   mask that persists across filters; peaks sorted to (filter, scan order).
// Phase 4: radial-shell collapse per peak.
// Record packing: RTHL > 0 (and z <= z_max on the lightcone), 11/33 floats.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "ppb_ctx.h"

namespace ppb {

namespace {

// ---------------------------------------------------------------------------
// device cosmology helpers (lightcone per-peak redshift, fcrit and D(z))
// ---------------------------------------------------------------------------
__device__ void dlinear_ab_dev(const DevCosmo& C, double ai, double* Dl, double* Da) {
  const int ntab = C.ng;
  if (ai > C.amin && ai < C.amax) {
    int jlo = 0, jhi = ntab + 1;
    while (jhi - jlo > 1) {
      const int jm = (jhi + jlo) / 2;
      if (ai > C.ga[jm - 1]) jlo = jm; else jhi = jm;
    }
    const int kk = jlo;
    int nl, kkl;
    if (kk < 2 || kk >= ntab) { nl = 2; kkl = kk - 1 > 1 ? kk - 1 : 1; } else { nl = 4; kkl = kk - 2; }
    const double* xa = C.ga + kkl - 1;
    const double* v1 = C.gD + kkl - 1;
    const double x = ai;
    double p1;
    if (nl == 4) {
      const double a1 = (x - xa[1]) / (xa[0] - xa[1]) * (x - xa[2]) / (xa[0] - xa[2]) * (x - xa[3]) / (xa[0] - xa[3]);
      const double a2 = (x - xa[0]) / (xa[1] - xa[0]) * (x - xa[2]) / (xa[1] - xa[2]) * (x - xa[3]) / (xa[1] - xa[3]);
      const double a3 = (x - xa[0]) / (xa[2] - xa[0]) * (x - xa[1]) / (xa[2] - xa[1]) * (x - xa[3]) / (xa[2] - xa[3]);
      const double a4 = (x - xa[0]) / (xa[3] - xa[0]) * (x - xa[1]) / (xa[3] - xa[1]) * (x - xa[2]) / (xa[3] - xa[2]);
      p1 = a1 * v1[0] + a2 * v1[1] + a3 * v1[2] + a4 * v1[3];
    } else {
      const double a1 = (x - xa[1]) / (xa[0] - xa[1]);
      p1 = a1 * v1[0] + (1.0 - a1) * v1[1];
    }
    *Dl = p1 * ai;
    *Da = p1;
  } else if (ai >= C.amax) {
    *Dl = C.D0 * ai; *Da = C.D0;
  } else {
    *Dl = C.Dinf * ai; *Da = C.Dinf;
  }
}

// chi_to_z (Cosmology.jl:155-169)
__device__ double chi_to_z_dev(const DevCosmo& C, double c) {
  if (c <= C.chis[0]) return 0.0;
  if (c >= C.chis[C.nchi - 1]) return C.chi_zmax;
  int lo = 1, hi = C.nchi;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (C.chis[mid - 1] <= c) lo = mid; else hi = mid;
  }
  const double zl = C.chi_zmax * (double)(lo - 1) / (double)(C.nchi - 1);
  const double zh = C.chi_zmax * (double)(hi - 1) / (double)(C.nchi - 1);
  const double fr = (c - C.chis[lo - 1]) / (C.chis[hi - 1] - C.chis[lo - 1]);
  return zl + fr * (zh - zl);
}

struct PrepArgs {
  const unsigned long long* keys;
  const uint32_t* vals;
  const float* ff;
  const float* lap;
  int npk;
  int n;
  double alatt;
  const double* fRf;
  const int32_t* fir2;
  const int32_t* fnp;        // per filter npart (rmax2rs > 0), else null
  int ievol;
  double z_out, fcrit0;
  double obs[3];
  DevCosmo C;
  int fbits;                 // key = ((tile << fbits | filter) << 40) | window-local flat index
  const double* tcen;        // 3 per tile: tile centre (null: all zero)
  int64_t* lin;
  double* Rf;
  int32_t* ir2;
  int32_t* np;
  double* Z;
  double* fc;
  float* FcRf;
  float* d2Rf;
  double* pos;   // 3 x npk
};

__global__ void prep_kernel(PrepArgs a) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.npk) return;
  const unsigned long long key = a.keys[q];
  const uint32_t slot = a.vals[q];
  const unsigned long long hi = key >> 40;
  const int f = (int)(hi & ((1ull << a.fbits) - 1));
  const int t = (int)(hi >> a.fbits);
  const int64_t lin = (int64_t)(key & ((1ull << 40) - 1));
  const int n = a.n;
  const int i = (int)(lin % n) + 1, j = (int)((lin / n) % n) + 1, k = (int)(lin / ((int64_t)n * n)) + 1;
  const double cen = 0.5 * (n + 1);
  // x = xbx + alatt (i - (n+1)/2) (PeakFind.jl:15-79; xbx = tile centre, 0 for run_tile)
  const double bx = a.tcen ? a.tcen[3 * t] : 0.0, by = a.tcen ? a.tcen[3 * t + 1] : 0.0,
               bz = a.tcen ? a.tcen[3 * t + 2] : 0.0;
  const double x = bx + a.alatt * (i - cen), y = by + a.alatt * (j - cen), z = bz + a.alatt * (k - cen);
  a.lin[q] = lin;
  a.Rf[q] = a.fRf[f];
  a.ir2[q] = a.fir2[f];
  if (a.fnp) a.np[q] = a.fnp[f];
  a.FcRf[q] = a.ff[slot];
  a.d2Rf[q] = a.lap[slot];
  a.pos[q] = x;
  a.pos[a.npk + q] = y;
  a.pos[2 * a.npk + q] = z;
  if (a.ievol == 1) {
    const double dx = x - a.obs[0], dy = y - a.obs[1], dz = z - a.obs[2];
    const double zpk = chi_to_z_dev(a.C, sqrt(dx * dx + dy * dy + dz * dz));
    const double ZZ = 1.0 + zpk;
    a.Z[q] = ZZ;
    double Dl, Da;
    dlinear_ab_dev(a.C, 1.0 / (1.0 + (ZZ - 1.0)), &Dl, &Da);
    a.fc[q] = 1.686 * Dl;
  } else {
    a.Z[q] = 1.0 + a.z_out;
    a.fc[q] = a.fcrit0;
  }
}

struct RecArgs {
  const double* res;
  const double* pos;
  const double* Rf;
  const float* FcRf;
  const float* d2Rf;
  const double* Z;
  int npk;
  int ievol;
  double z_max;
  double alatt;
  double Omnr, OL;
  int ilpt;
  int nf;
  DevCosmo C;
  int* flags;
  const int* offs;
  float* rec;
  float* rthl;   // per record RTHL (for the max)
};

__global__ void flag_kernel(RecArgs a) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.npk) return;
  const double R = a.res[(int64_t)q * RES_N];
  bool ok = R > 0.0;
  if (a.ievol == 1 && a.Z[q] - 1.0 > a.z_max) ok = false;
  a.flags[q] = ok ? 1 : 0;
}

// record layout: Pipeline.jl:263-306, Catalog.jl:26-46
__global__ void record_kernel(RecArgs a) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.npk || !a.flags[q]) return;
  const double* r = a.res + (int64_t)q * RES_N;
  const double ZZ = a.Z[q];
  const double a_pk = 1.0 / ZZ;
  double Dl, Dpk;
  dlinear_ab_dev(a.C, a_pk, &Dl, &Dpk);   // third return value of Dlinear_ab (Pipeline.jl:259)
  double v2f = 0.0;
  if (a.ilpt >= 2) {
    const double a3 = a_pk * a_pk * a_pk;
    const double Oma = a.Omnr * a3 / (a.Omnr * a3 + a.OL);
    v2f = -(-3.0 / 7.0 * pow(Oma, -1.0 / 143) * (Dpk * Dpk));
  }
  float* o = a.rec + (int64_t)a.offs[q] * a.nf;
  o[0] = (float)a.pos[q];
  o[1] = (float)a.pos[a.npk + q];
  o[2] = (float)a.pos[2 * a.npk + q];
  for (int L = 0; L < 3; L++) o[3 + L] = (float)(r[2 + L] * Dpk);
  const float RTHLp = (float)(r[0] * a.alatt);
  o[6] = RTHLp;
  for (int L = 0; L < 3; L++) o[7 + L] = (float)(r[5 + L] * v2f);
  o[10] = (float)r[23];
  a.rthl[a.offs[q]] = RTHLp;
  if (a.nf == 33) {
    const double* s = r + 8;   // column-major strain
    o[11] = (float)r[24];
    o[12] = (float)r[25];
    o[13] = (float)s[0];
    o[14] = (float)s[4];
    o[15] = (float)s[8];
    o[16] = (float)s[1 + 3 * 2];
    o[17] = (float)s[0 + 3 * 2];
    o[18] = (float)s[0 + 3 * 1];
    o[19] = (float)r[30];
    o[20] = (float)r[26];
    for (int L = 0; L < 3; L++) {
      o[21 + L] = (float)r[17 + L];
      o[24 + L] = (float)r[27 + L];
    }
    o[27] = (float)a.Rf[q];
    o[28] = a.FcRf[q];
    o[29] = a.d2Rf[q];
    for (int L = 0; L < 3; L++) o[30 + L] = (float)r[20 + L];
  }
}

// sorted peak keys -> 1-based (i, j, k), ipp and filter number
__global__ void unpack_peaks_kernel(const unsigned long long* keys, int npk, int n, int fbits, int32_t* ijk,
                                    int64_t* ipp, int32_t* filt) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= npk) return;
  const unsigned long long key = keys[q];
  const int64_t lin = (int64_t)(key & ((1ull << 40) - 1));
  ijk[q] = (int32_t)(lin % n) + 1;
  ijk[npk + q] = (int32_t)((lin / n) % n) + 1;
  ijk[2 * npk + q] = (int32_t)(lin / ((int64_t)n * n)) + 1;
  ipp[q] = lin + 1;
  filt[q] = (int32_t)((key >> 40) & ((1ull << fbits) - 1)) + 1;
}

__global__ void tile_count_kernel(const unsigned long long* keys, int npk, int shift, int* counts) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < npk) atomicAdd(counts + (int)(keys[q] >> shift), 1);
}

}  // namespace

// ---------------------------------------------------------------------------
// plans and buffers for one grid size
// ---------------------------------------------------------------------------
static cufftHandle make_plan(int n, cufftType t, int batch) {
  cufftHandle h;
  int dims[3] = {n, n, n};
  PPB_CUFFT(cufftPlanMany(&h, 3, dims, nullptr, 1, 0, nullptr, 1, 0, t, batch));
  return h;
}

TileRes::~TileRes() {
  for (auto& g : graphs)   // before the plans whose kernels they launch
    if (g.second) cudaGraphExecDestroy(g.second);
  graphs.clear();
  for (cufftHandle h : {r2c, c2r1, c2r2, c2r3, c2r6, yz1, yz2})
    if (h) cufftDestroy(h);
}

void TileRes::setup(int nn, cudaStream_t s) {
  if (n == nn) return;
  for (cufftHandle* h : {&r2c, &c2r1, &c2r2, &c2r3, &c2r6, &yz1, &yz2})
    if (*h) { cufftDestroy(*h); *h = 0; }
  n = nn;
  const int64_t N = (int64_t)n * n * n, M = (int64_t)(n / 2 + 1) * n * n;
  r2c = make_plan(n, CUFFT_R2C, 1);
  c2r1 = make_plan(n, CUFFT_C2R, 1);
  c2r2 = make_plan(n, CUFFT_C2R, 2);
  c2r3 = make_plan(n, CUFFT_C2R, 3);
  c2r6 = make_plan(n, CUFFT_C2R, 6);
  for (cufftHandle h : {r2c, c2r1, c2r2, c2r3, c2r6}) PPB_CUFFT(cufftSetStream(h, s));

  delta.ensure(N * 4);
  dk.ensure(M * 8);
  psi.ensure(3 * N * 4);
  psi2.ensure(3 * N * 4);
  lapd.ensure(N * 4);
  kw.ensure(6 * M * 8);
  rw.ensure(6 * N * 4);
  mask.ensure(N);
  count.ensure(64);
}

size_t TileRes::bytes() const {
  size_t b = 0;
  for (const DevBuf* d : {&delta, &dk, &psi, &psi2, &lapd, &aos, &kw, &rw, &mask, &count, &wtab, &keys, &vals, &ff,
                          &lap, &keys_s, &vals_s, &tmp, &p_lin, &p_Rf, &p_ir2, &p_np, &p_Z, &p_fc, &p_FcRf, &p_d2Rf,
                          &p_pos, &res, &flags, &offs, &rec, &rthl, &xtw})
    b += d->bytes;
  return b;
}

void TileRes::setup_fused(cudaStream_t s) {
  if (yz1) return;
  int dims[2] = {n, n};
  const int nh = n / 2 + 1;
  PPB_CUFFT(cufftPlanMany(&yz1, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2C, nh));
  PPB_CUFFT(cufftPlanMany(&yz2, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2C, 2 * nh));
  for (cufftHandle h : {yz1, yz2}) PPB_CUFFT(cufftSetStream(h, s));
  xpeak_prepare(n);
  xtw.ensure((size_t)n * sizeof(float2));
}

void TileRes::ensure_peaks(int64_t c) {
  if (c <= cap) return;
  cap = c;
  keys.ensure(cap * 8);
  vals.ensure(cap * 4);
  ff.ensure(cap * 4);
  lap.ensure(cap * 4);
  keys_s.ensure(cap * 8);
  vals_s.ensure(cap * 4);
  p_lin.ensure(cap * 8);
  p_Rf.ensure(cap * 8);
  p_ir2.ensure(cap * 4);
  p_np.ensure(cap * 4);
  p_Z.ensure(cap * 8);
  p_fc.ensure(cap * 8);
  p_FcRf.ensure(cap * 4);
  p_d2Rf.ensure(cap * 4);
  p_pos.ensure(cap * 24);
  res.ensure(cap * RES_N * 8);
  flags.ensure(cap * 4 + 4);
  offs.ensure(cap * 4 + 4);
  rec.ensure(cap * 33 * 4);
  rthl.ensure(cap * 4);
  size_t t1 = 0, t2 = 0;
  PPB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t1, keys.as<unsigned long long>(), keys_s.as<unsigned long long>(),
                                           vals.as<uint32_t>(), vals_s.as<uint32_t>(), (int)cap, 0, 64));
  PPB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t2, flags.as<int>(), offs.as<int>(), (int)cap + 1));
  size_t t3 = 0;
  PPB_CUDA(cub::DeviceReduce::Max(nullptr, t3, rthl.as<float>(), rthl.as<float>(), (int)cap));
  tmp.ensure(std::max(std::max(t1, t2), t3) + 256);
}

// ---------------------------------------------------------------------------
// the pipeline
// ---------------------------------------------------------------------------
void check_params(const ppb_tile_params* p, const double* Rf, int nfilt) {
  PPB_REQUIRE(p != nullptr, "params is null");
  PPB_REQUIRE(p->n >= 8 && p->n <= 2048, "n must be in [8, 2048]");
  PPB_REQUIRE(p->boxsize > 0, "boxsize must be positive");
  PPB_REQUIRE(p->nbuff >= 2 && 2 * p->nbuff < p->n, "nbuff must satisfy 2 <= nbuff and 2 nbuff < n");
  PPB_REQUIRE(Rf != nullptr && nfilt >= 1 && nfilt <= 4096, "need 1..4096 filter radii");
  for (int i = 0; i < nfilt; i++) PPB_REQUIRE(Rf[i] > 0, "filter radii must be positive");
  PPB_REQUIRE(p->ilpt == 1 || p->ilpt == 2, "ilpt must be 1 or 2");
  PPB_REQUIRE(p->wsmooth == 0 || p->wsmooth == 1 || p->wsmooth == 3, "wsmooth must be 0, 1 or 3");
  PPB_REQUIRE(p->ievol == 0 || p->ievol == 1, "ievol must be 0 or 1");
  PPB_REQUIRE(p->pk_scale >= 0.0, "pk_scale must be >= 0 (0 means 1)");
  PPB_REQUIRE(p->rmax2rs >= 0.0 && p->rmax2rs <= 1e6, "rmax2rs must be in [0, 1e6]");
}

uint64_t tile_footprint(const ppb_tile_params* p) { return tile_bytes_estimate(p->n) + shell_bytes_estimate(p->n); }

// Peak buffers of a grid of N cells before the first run: one peak per 40
// cells.  The 384^3 benchmark tile has one per 66 cells at sigma8 0.808 and
// about 10 % more at 0.85; starting with room for them means a served stream
// of varying sigma8 does not grow the buffers (every cudaFree of a growth
// waits for all slots' work on the device).  A larger count still grows them.
int64_t initial_peak_capacity(int64_t N) { return std::max<int64_t>(1 << 16, std::min<int64_t>(N / 40, 1 << 22)); }

uint64_t tile_bytes_estimate(int nn) {
  const uint64_t n = (uint64_t)nn, N = n * n * n, M = (n / 2 + 1) * n * n;
  // TileRes fields: delta, psi (3), psi2 (3), lapd, rw (6), mask, aos (8 floats), dk + kw (7 complex)
  const uint64_t fields = N * 4 * (1 + 3 + 3 + 1 + 6) + N + N * 32 + M * 8 * 7;
  // peak, result and record buffers: initial_peak_capacity (1/40 peak per
  // cell), 0.5 KB each; plans and their work areas
  return fields + N * 13 + ((uint64_t)64 << 20);
}

uint64_t shell_bytes_estimate(int nn) {
  const uint64_t n = (uint64_t)nn, N = n * n * n;
  // the shell stage's per-warp staging rows (16 warps per SM, 600 shells of
  // 24 doubles) and the profile pool (about 100 bytes per cell)
  return (uint64_t)148 * 16 * 600 * 24 * 8 + N * 100;
}

namespace {

// host state of one run shared by the phases
struct Run {
  ppb_ctx* ctx;
  Slot* sl;
  const ppb_tile_params* p;
  cudaStream_t s;
  Launch L;
  double Om, alatt;
  bool plain, want_lap;
  std::vector<double> Rf;   // descending
  int nfilt, fbits;
  const GrowthTable* G;
  double fcrit_val;
  int nhunt;
  ShellTable* shells;
  DevCosmo C;
  bool npcap;   // rmax2rs > 0: per-peak cell caps (filt_np, p_np)
  // peak search of a caller's field (ppb_peak_find_tile): fcrit per filter
  // (empty: the window's), and the mask as the caller gave it (else zeroed)
  std::vector<float> ffc;
  bool keep_mask = false;
  const void* mask_src = nullptr;   // keep_mask: the caller's mask (host or device), copied in per attempt
};

// a peak-search window: a tile of nm^3 cells at `off` in the field grid
struct Win {
  int64_t off;
  float fcrit;
};

void setup_run(Run& r, ppb_ctx* ctx, Slot& sl, const ppb_tile_params* p, const double* Rf_in, int nfilt,
               double alatt) {
  r.ctx = ctx;
  r.sl = &sl;
  r.p = p;
  r.s = sl.stream;
  r.L = Launch{sl.stream, &sl.launches};
  r.Om = p->Omx + p->OmB;
  r.alatt = alatt;
  r.plain = p->plain != 0;
  r.want_lap = p->ioutshear >= 1;
  r.Rf.assign(Rf_in, Rf_in + nfilt);
  std::stable_sort(r.Rf.begin(), r.Rf.end(), [](double a, double b) { return a > b; });
  r.nfilt = nfilt;
  r.fbits = 1;
  while ((1 << r.fbits) < nfilt) r.fbits++;
  r.G = &ctx->growth(r.Om, p->OmB, p->Omvac, p->h);
  r.fcrit_val = fsc_of_z(*r.G, p->z_out);
  r.nhunt = std::min(p->nbuff - 1, (int)std::floor(r.Rf[0] * 1.75 / alatt));
  PPB_REQUIRE(r.nhunt >= 1, "nhunt = min(nbuff-1, floor(1.75 Rfmax/alatt)) must be >= 1");
  r.shells = &ctx->shell_table(r.nhunt, r.s);
  // rmax2rs > 0 (RadialShell.jl:288-295): a peak of filter radius Rf uses the
  // first npart = min(floor(4/3 pi (rmax2rs Rf / alatt)^3), npartmax) cells
  // of the shell list.  The pre-mask test of :310-316 needs no counterpart:
  // it can only skip a peak whose filter has floor(rmax2rs Rf / alatt) = 0,
  // i.e. npart <= 4 cells, which closes no shell beyond the centre (the six
  // r^2 = 1 cells end at cell 7), so the peak reaches m0 = 1 and returns
  // no_collapse (:650-653) whether or not it is skipped.  The result is then
  // independent of the order in which peaks write and read the mask.
  r.npcap = p->rmax2rs > 0.0;
  if (r.npcap) {
    const double f3p = 4.0 / 3.0 * 3.141592653589793;
    std::vector<int32_t> fnp(nfilt);
    for (int f = 0; f < nfilt; f++) {
      const double x = p->rmax2rs * r.Rf[f] / alatt;
      const double v = f3p * (x * x * x);
      fnp[f] = v >= (double)r.shells->ncells ? (int32_t)r.shells->ncells : (int32_t)std::floor(v);
    }
    sl.filt_np.ensure(nfilt * 4);
    PPB_CUDA(cudaMemcpyAsync(sl.filt_np.p, fnp.data(), nfilt * 4, cudaMemcpyHostToDevice, r.s));
  }
  std::vector<int32_t> fir2(nfilt);
  for (int f = 0; f < nfilt; f++)
    fir2[f] = (int32_t)std::min(std::floor((1.75 * r.Rf[f] / alatt) * (1.75 * r.Rf[f] / alatt)),
                                std::floor((40.0 / alatt - 1) * (40.0 / alatt - 1)));
  r.C = ctx->dev_cosmo(sl, *r.G, r.Om, p->Omvac, p->h, p->ievol == 1 ? p->z_max + 1.0 : 0.0, p->ievol == 1);
  sl.filt_Rf.ensure(nfilt * 8);
  sl.filt_ir2.ensure(nfilt * 4);
  PPB_CUDA(cudaMemcpyAsync(sl.filt_Rf.p, r.Rf.data(), nfilt * 8, cudaMemcpyHostToDevice, r.s));
  PPB_CUDA(cudaMemcpyAsync(sl.filt_ir2.p, fir2.data(), nfilt * 4, cudaMemcpyHostToDevice, r.s));
}

// phase 1 (Pipeline.jl:90-140, MultiTile.jl:157-194): Threefry noise -> R2C
// -> sqrt(P) -> C2R = delta; delta_k = R2C(delta), projected Hermitian;
// 1LPT, 2LPT and the Laplacian field, all on the n^3 grid of `box`
void fields_phase(Run& r, TileRes& T, int n, double box) {
  const ppb_tile_params* p = r.p;
  const Launch& L = r.L;
  const int64_t N = (int64_t)n * n * n, M = (int64_t)(n / 2 + 1) * n * n;
  const double inv_n3 = 1.0 / (double)N;
  float2* dkp = T.dk.as<float2>();
  float2* kw = T.kw.as<float2>();
  float* rw = T.rw.as<float>();
  const Shared& sh = r.ctx->sh;
  launch_noise(L, rw, n, p->seed);
  PPB_CUFFT(cufftExecR2C(T.r2c, rw, (cufftComplex*)kw));
  launch_convolve(L, kw, n, box, sh.pk_lk.as<double>(), sh.pk_lp.as<double>(), sh.pk_n,
                  p->pk_scale > 0.0 ? p->pk_scale : 1.0, inv_n3);
  launch_hermitise(L, kw, n, 1);
  PPB_CUFFT(cufftExecC2R(T.c2r1, (cufftComplex*)kw, T.delta.as<cufftReal>()));
  PPB_CUFFT(cufftExecR2C(T.r2c, T.delta.as<cufftReal>(), (cufftComplex*)dkp));
  // one Hermitian projection of delta_k: every filter output W(|k|) delta_k
  // (and k^2 W delta_k) is then Hermitian as it stands
  launch_hermitise(L, dkp, n, 1);
  // 1LPT
  launch_lpt1(L, dkp, kw, n, box, inv_n3);
  launch_hermitise(L, kw, n, 3);
  if (r.plain) {
    for (int c = 0; c < 3; c++)
      PPB_CUFFT(cufftExecC2R(T.c2r1, (cufftComplex*)(kw + c * M), T.psi.as<cufftReal>() + c * N));
  } else {
    PPB_CUFFT(cufftExecC2R(T.c2r3, (cufftComplex*)kw, T.psi.as<cufftReal>()));
  }
  // 2LPT
  if (p->ilpt >= 2) {
    launch_phi(L, dkp, kw, n, box, inv_n3);
    launch_hermitise(L, kw, n, 6);
    if (r.plain) {
      for (int c = 0; c < 6; c++) PPB_CUFFT(cufftExecC2R(T.c2r1, (cufftComplex*)(kw + c * M), rw + c * N));
    } else {
      PPB_CUFFT(cufftExecC2R(T.c2r6, (cufftComplex*)kw, rw));
    }
    launch_src2(L, rw, T.lapd.as<float>(), N);   // lapd buffer as scratch for src2
    PPB_CUFFT(cufftExecR2C(T.r2c, T.lapd.as<cufftReal>(), (cufftComplex*)kw));
    launch_lpt2(L, kw, kw + M, n, box, inv_n3);
    launch_hermitise(L, kw + M, n, 3);
    if (r.plain) {
      for (int c = 0; c < 3; c++)
        PPB_CUFFT(cufftExecC2R(T.c2r1, (cufftComplex*)(kw + (1 + c) * M), T.psi2.as<cufftReal>() + c * N));
    } else {
      PPB_CUFFT(cufftExecC2R(T.c2r3, (cufftComplex*)(kw + M), T.psi2.as<cufftReal>()));
    }
  }
  // Laplacian field (Pipeline.jl:35-51): irfft(k^2 delta_k) / n^3
  if (r.want_lap) {
    launch_lapd(L, dkp, kw, n, box, (float)(inv_n3 * inv_n3));
    launch_hermitise(L, kw, n, 1);
    PPB_CUFFT(cufftExecC2R(T.c2r1, (cufftComplex*)kw, T.lapd.as<cufftReal>()));
  }
}

// phase 2 (Pipeline.jl:144-196, MultiTile.jl:218-275): per filter, largest
// first, the smoothed field (and its k^2-weighted twin) on the n^3 grid, then
// the peak search in every window (mask shared: windows search disjoint
// cores).  Keys (window, filter, window-local index) restore the reference's
// order.  Returns the number of peaks in T's peak buffers.
int64_t peaks_phase(Run& r, TileRes& T, int n, double box, const std::vector<Win>& wins, int nm) {
  const ppb_tile_params* p = r.p;
  const Launch& L = r.L;
  const int64_t N = (int64_t)n * n * n, M = (int64_t)(n / 2 + 1) * n * n;
  const double inv_n3 = 1.0 / (double)N;
  float2* dkp = T.dk.as<float2>();
  float2* kw = T.kw.as<float2>();
  float* rw = T.rw.as<float>();
  const int qn = window_table_size(n);
  T.wtab.ensure((size_t)r.nfilt * 2 * qn * sizeof(float));
  // one window over the whole grid (run_tile and the split's tiles; the
  // multi-tile run searches several windows of one global grid) and a
  // supported size: the x pass of each filter's transform runs fused with the
  // peak search.  By default only with the k^2-weighted twin (two fields)
  // and n = 64 J, J = 3, 5, 6, 7: there cuFFT's 3-D C2R is the slow part
  // (peaks stage 384^3 26.8 -> 20.5 ms, 448^3 49.7 -> 40.0, 320^3 14.7 ->
  // 12.1); for J a power of two (256^3 4.78 / 4.75, 512^3 46.4 / 50.4) and
  // for one field (the split's tiles) the full transforms are as fast or faster
  const int fx = r.ctx->sh.fused_x.load();
  const int J = n / 64;
  const bool fused = !r.plain && (fx == 1 || (fx == -1 && r.want_lap && (J & (J - 1)) != 0)) &&
                     xpeak_supported(n, p->nbuff) && wins.size() == 1 && wins[0].off == 0 && nm == n;
  if (fused) T.setup_fused(r.s);
  int64_t npk = 0;
  for (int attempt = 0; attempt < 2; attempt++) {
    PeakBuf pb{T.keys.as<unsigned long long>(), T.vals.as<uint32_t>(), T.ff.as<float>(), T.lap.as<float>(),
               T.count.as<int>(), T.cap};
    if (r.keep_mask) PPB_CUDA(cudaMemcpyAsync(T.mask.p, r.mask_src, N, cudaMemcpyDefault, r.s));
    // the whole filter bank as one graph (window tables, per filter the
    // window multiply, the inverse transforms and the peak search)
    r.ctx->captured(*r.sl, T.graphs, r.keep_mask ? 3 : 1, (int64_t)n * 4096 + (int64_t)wins.size(), [&] {
      if (!r.keep_mask) PPB_CUDA(cudaMemsetAsync(T.mask.p, 0, N, r.s));
      PPB_CUDA(cudaMemsetAsync(T.count.p, 0, 64, r.s));
      launch_window_tables(L, T.wtab.as<float>(), n, box, r.sl->filt_Rf.as<double>(), r.nfilt, p->wsmooth,
                           r.want_lap);
      if (fused) launch_twiddles(L, T.xtw.as<float2>(), n);
      for (int f = 0; f < r.nfilt; f++) {
        float2* o1 = r.want_lap ? kw + M : nullptr;
        if (fused) {
          // window multiply into [kx][kz][ky], z and y by cuFFT (both fields
          // in one call), then x and the peak search in one kernel
          launch_window_t(L, dkp, kw, o1, n, T.wtab.as<float>() + (size_t)f * 2 * qn, inv_n3);
          PPB_CUFFT(cufftExecC2C(o1 ? T.yz2 : T.yz1, (cufftComplex*)kw, (cufftComplex*)kw, CUFFT_INVERSE));
          launch_xpeak(L, kw, o1, T.xtw.as<float2>(), T.mask.as<uint8_t>(), T.count.as<unsigned>() + 2, n,
                       p->nbuff, r.ffc.empty() ? wins[0].fcrit : r.ffc[f], (unsigned long long)f, pb);
          continue;
        }
        launch_window(L, dkp, kw, o1, n, T.wtab.as<float>() + (size_t)f * 2 * qn, inv_n3);
        if (r.want_lap && !r.plain) {
          PPB_CUFFT(cufftExecC2R(T.c2r2, (cufftComplex*)kw, rw));
        } else {
          PPB_CUFFT(cufftExecC2R(T.c2r1, (cufftComplex*)kw, rw));
          if (r.want_lap) PPB_CUFFT(cufftExecC2R(T.c2r1, (cufftComplex*)(kw + M), rw + N));
        }
        for (size_t t = 0; t < wins.size(); t++) {
          const Win& w = wins[t];
          launch_peakfind(L, rw + w.off, r.want_lap ? rw + N + w.off : nullptr, T.mask.as<uint8_t>() + w.off, nm,
                          nm, nm, n, (int64_t)n * n, p->nbuff, r.ffc.empty() ? w.fcrit : r.ffc[f],
                          ((unsigned long long)t << r.fbits) | (unsigned long long)f, pb);
        }
      }
    });
    int cnt = 0;
    PPB_CUDA(cudaMemcpyAsync(&cnt, T.count.p, 4, cudaMemcpyDeviceToHost, r.s));
    PPB_CUDA(cudaStreamSynchronize(r.s));
    npk = cnt;
    if (npk <= T.cap) break;
    PPB_REQUIRE(attempt == 0, "peak capacity exceeded twice");
    T.ensure_peaks((int64_t)(npk * 1.25) + 1024);   // grow and redo the filter bank
  }
  return npk;
}

// sort the peaks to (window, filter, scan order) and derive the per-peak
// parameters; tcen (device, 3 per window) gives the window centres
void prep_phase(Run& r, TileRes& T, int64_t npk, int nm, int nwin, const double* tcen) {
  if (npk <= 0) return;
  int tbits = 0;
  while ((1 << tbits) < nwin) tbits++;
  size_t tb = T.tmp.bytes;
  PPB_CUDA(cub::DeviceRadixSort::SortPairs(T.tmp.p, tb, T.keys.as<unsigned long long>(),
                                           T.keys_s.as<unsigned long long>(), T.vals.as<uint32_t>(),
                                           T.vals_s.as<uint32_t>(), (int)npk, 0, 40 + r.fbits + tbits, r.s));
  r.sl->launches++;
  const ppb_tile_params* p = r.p;
  PrepArgs pa{};
  pa.keys = T.keys_s.as<unsigned long long>();
  pa.vals = T.vals_s.as<uint32_t>();
  pa.ff = T.ff.as<float>();
  pa.lap = T.lap.as<float>();
  pa.npk = (int)npk;
  pa.n = nm;
  pa.alatt = r.alatt;
  pa.fRf = r.sl->filt_Rf.as<double>();
  pa.fir2 = r.sl->filt_ir2.as<int32_t>();
  pa.ievol = p->ievol;
  pa.z_out = p->z_out;
  pa.fcrit0 = r.fcrit_val;
  pa.obs[0] = p->cenx; pa.obs[1] = p->ceny; pa.obs[2] = p->cenz;
  pa.C = r.C;
  pa.fbits = r.fbits;
  pa.tcen = tcen;
  pa.lin = T.p_lin.as<int64_t>();
  pa.Rf = T.p_Rf.as<double>();
  pa.ir2 = T.p_ir2.as<int32_t>();
  pa.fnp = r.npcap ? r.sl->filt_np.as<int32_t>() : nullptr;
  pa.np = T.p_np.as<int32_t>();
  pa.Z = T.p_Z.as<double>();
  pa.fc = T.p_fc.as<double>();
  pa.FcRf = T.p_FcRf.as<float>();
  pa.d2Rf = T.p_d2Rf.as<float>();
  pa.pos = T.p_pos.as<double>();
  prep_kernel<<<(unsigned)((npk + 255) / 256), 256, 0, r.s>>>(pa);
  PPB_LAUNCHED(r.sl->launches);
}

// phase 4 (Pipeline.jl:200-240) for peaks [p0, p1) on an nm^3 window whose
// packed records are aos (and Laplacian lapd)
void shells_phase(Run& r, TileRes& T, int64_t p0, int64_t p1, int nm, const float4* aos, const float* lapd,
                  ShellStats* acc, const std::function<void()>& pre = nullptr) {
  if (p1 <= p0) return;
  ShellArgs a = r.ctx->shell_args(*r.sl, *r.shells, nm, r.alatt, aos, lapd);
  a.pk = PeakParams{T.p_lin.as<int64_t>() + p0, T.p_Rf.as<double>() + p0, T.p_ir2.as<int32_t>() + p0,
                    T.p_Z.as<double>() + p0, T.p_fc.as<double>() + p0};
  a.npk = p1 - p0;
  a.npcap = r.npcap ? T.p_np.as<int32_t>() + p0 : nullptr;
  a.out = T.res.as<double>() + p0 * RES_N;
  ShellStats st{};
  r.ctx->run_shells(*r.sl, a, !r.plain, !r.plain, &st, pre);
  acc->visits += st.visits;
  acc->guard += st.guard;
  acc->akk += st.akk;
  for (int i = 0; i < 5; i++) acc->dump[i] += st.dump[i];
  for (int i = 0; i < 16; i++) acc->raw[i] += st.raw[i];
  acc->ms += st.ms;
  for (int i = 0; i < 4; i++) acc->kms[i] += st.kms[i];
  acc->pool_rows += st.pool_rows;
  acc->batches += st.batches;
}

// records (Pipeline.jl:243-318): RTHL > 0 (and z <= z_max on the lightcone),
// 11 or 33 floats in peak order, and their largest RTHL
void records_phase(Run& r, TileRes& T, int64_t npk, int64_t* nrec_out, float* rmax_out) {
  const ppb_tile_params* p = r.p;
  const int nf = p->ioutshear >= 1 ? 33 : 11;
  int64_t nrec = 0;
  float rmax = 0.f;
  if (npk > 0) {
    RecArgs a{};
    a.res = T.res.as<double>();
    a.pos = T.p_pos.as<double>();
    a.Rf = T.p_Rf.as<double>();
    a.FcRf = T.p_FcRf.as<float>();
    a.d2Rf = T.p_d2Rf.as<float>();
    a.Z = T.p_Z.as<double>();
    a.npk = (int)npk;
    a.ievol = p->ievol;
    a.z_max = p->z_max;
    a.alatt = r.alatt;
    a.Omnr = r.Om;
    a.OL = p->Omvac;
    a.ilpt = p->ilpt;
    a.nf = nf;
    a.C = r.C;
    a.flags = T.flags.as<int>();
    a.offs = T.offs.as<int>();
    a.rec = T.rec.as<float>();
    a.rthl = T.rthl.as<float>();
    const unsigned gb = (unsigned)((npk + 255) / 256);
    flag_kernel<<<gb, 256, 0, r.s>>>(a);
    PPB_LAUNCHED(r.sl->launches);
    PPB_CUDA(cudaMemsetAsync(T.flags.as<int>() + npk, 0, 4, r.s));
    size_t tb = T.tmp.bytes;
    PPB_CUDA(cub::DeviceScan::ExclusiveSum(T.tmp.p, tb, T.flags.as<int>(), T.offs.as<int>(), (int)npk + 1, r.s));
    r.sl->launches++;
    record_kernel<<<gb, 256, 0, r.s>>>(a);
    PPB_LAUNCHED(r.sl->launches);
    int nr = 0;
    PPB_CUDA(cudaMemcpyAsync(&nr, T.offs.as<int>() + npk, 4, cudaMemcpyDeviceToHost, r.s));
    PPB_CUDA(cudaStreamSynchronize(r.s));
    nrec = nr;
    if (nrec > 0) {
      size_t tb2 = T.tmp.bytes;
      float* dmax = T.count.as<float>() + 8;
      PPB_CUDA(cub::DeviceReduce::Max(T.tmp.p, tb2, T.rthl.as<float>(), dmax, (int)nrec, r.s));
      r.sl->launches++;
      PPB_CUDA(cudaMemcpyAsync(&rmax, dmax, 4, cudaMemcpyDeviceToHost, r.s));
    }
  }
  PPB_CUDA(cudaStreamSynchronize(r.s));
  *nrec_out = nrec;
  *rmax_out = nrec > 0 ? rmax : 0.f;
}

void check_shell_stats(const ShellStats& st) {
  if (st.guard != 0)
    throw Error{PPB_ERR_CUDA, "shell truncation guard tripped: a profile read beyond the gathered shells"};
  if (st.akk != 0)
    throw Error{PPB_ERR_INVALID, "kernel_strain SPH table index out of range (the reference raises here too)"};
}

}  // namespace

void peak_find_tile_core(ppb_ctx* ctx, Slot& sl, const float* delta, int n, const double* Rf, const double* fcrit,
                         int nfilt, int8_t* mask, double xbx, double ybx, double zbx, double alatt, int nbuff,
                         int wsmooth, int ioutshear, const PeakTileOut& o) {
  PPB_REQUIRE(delta && Rf && fcrit && mask && o.npeaks, "null argument");
  PPB_REQUIRE(n >= 8 && n <= 2048, "n must be in [8, 2048]");
  PPB_REQUIRE(alatt > 0.0, "alatt must be positive");
  PPB_REQUIRE(nbuff >= 1 && 2 * nbuff < n, "nbuff must satisfy 1 <= nbuff and 2 nbuff < n");
  PPB_REQUIRE(nfilt >= 1 && nfilt <= 4096, "need 1..4096 filters");
  for (int f = 0; f < nfilt; f++) PPB_REQUIRE(Rf[f] > 0.0, "filter radii must be positive");
  PPB_REQUIRE(wsmooth == 0 || wsmooth == 1 || wsmooth == 3, "wsmooth must be 0, 1 or 3");
  PPB_REQUIRE(o.capacity >= 0, "capacity must be >= 0");
  const int64_t N = (int64_t)n * n * n;
  // the tile's own periodic box, boxsize_local = n alatt (ext/CUDAExt.jl:3081)
  ppb_tile_params p{};
  p.n = n;
  p.boxsize = n * alatt;
  p.nbuff = nbuff;
  p.wsmooth = wsmooth;
  p.ioutshear = ioutshear;
  p.ilpt = 1;
  Run r{};
  r.ctx = ctx;
  r.sl = &sl;
  r.p = &p;
  r.s = sl.stream;
  r.L = Launch{sl.stream, &sl.launches};
  r.alatt = alatt;
  r.plain = false;
  r.want_lap = ioutshear >= 1;
  r.Rf.assign(Rf, Rf + nfilt);   // the caller's order (the filter loop of ext/CUDAExt.jl:3118)
  r.nfilt = nfilt;
  r.fbits = 1;
  while ((1 << r.fbits) < nfilt) r.fbits++;
  r.ffc.resize(nfilt);
  for (int f = 0; f < nfilt; f++) r.ffc[f] = (float)fcrit[f];   // find_peaks compares in Float32
  r.keep_mask = true;
  r.mask_src = mask;
  r.npcap = false;
  sl.filt_Rf.ensure(nfilt * 8);
  sl.filt_ir2.ensure(nfilt * 4);
  PPB_CUDA(cudaMemcpyAsync(sl.filt_Rf.p, r.Rf.data(), nfilt * 8, cudaMemcpyHostToDevice, r.s));
  PPB_CUDA(cudaMemsetAsync(sl.filt_ir2.p, 0, nfilt * 4, r.s));
  TileRes& T = sl.tile_for(n);
  T.setup(n, r.s);
  if (T.cap == 0) T.ensure_peaks(initial_peak_capacity(N));
  // rfft(delta) once, projected Hermitian as run_tile's delta_k
  PPB_CUDA(cudaMemcpyAsync(T.delta.p, delta, N * 4, cudaMemcpyDefault, r.s));
  PPB_CUFFT(cufftExecR2C(T.r2c, T.delta.as<cufftReal>(), T.dk.as<cufftComplex>()));
  launch_hermitise(r.L, T.dk.as<float2>(), n, 1);
  const int64_t npk = peaks_phase(r, T, n, p.boxsize, {Win{0, 0.f}}, n);
  *o.npeaks = npk;
  if (npk > o.capacity) {
    PPB_CUDA(cudaStreamSynchronize(r.s));
    throw Error{PPB_ERR_CAPACITY, "peak output capacity too small; *npeaks holds the count needed"};
  }
  sl.tcen.ensure(3 * 8);
  const double cen[3] = {xbx, ybx, zbx};
  PPB_CUDA(cudaMemcpyAsync(sl.tcen.p, cen, 24, cudaMemcpyHostToDevice, r.s));
  if (npk > 0) {
    prep_phase(r, T, npk, n, 1, sl.tcen.as<double>());
    sl.pft.ensure((size_t)npk * 24);
    int32_t* ijk = sl.pft.as<int32_t>();
    int64_t* ipp = reinterpret_cast<int64_t*>(sl.pft.as<char>() + (size_t)npk * 16);
    int32_t* filt = ijk + 3 * npk;
    unpack_peaks_kernel<<<(unsigned)((npk + 255) / 256), 256, 0, r.s>>>(T.keys_s.as<unsigned long long>(), (int)npk,
                                                                        n, r.fbits, ijk, ipp, filt);
    PPB_LAUNCHED(sl.launches);
    const size_t b4 = (size_t)npk * 4, b8 = (size_t)npk * 8;
    if (o.pi) PPB_CUDA(cudaMemcpyAsync(o.pi, ijk, b4, cudaMemcpyDefault, r.s));
    if (o.pj) PPB_CUDA(cudaMemcpyAsync(o.pj, ijk + npk, b4, cudaMemcpyDefault, r.s));
    if (o.pk) PPB_CUDA(cudaMemcpyAsync(o.pk, ijk + 2 * npk, b4, cudaMemcpyDefault, r.s));
    if (o.ipp) PPB_CUDA(cudaMemcpyAsync(o.ipp, ipp, b8, cudaMemcpyDefault, r.s));
    if (o.filter) PPB_CUDA(cudaMemcpyAsync(o.filter, filt, b4, cudaMemcpyDefault, r.s));
    if (o.x) PPB_CUDA(cudaMemcpyAsync(o.x, T.p_pos.as<double>(), b8, cudaMemcpyDefault, r.s));
    if (o.y) PPB_CUDA(cudaMemcpyAsync(o.y, T.p_pos.as<double>() + npk, b8, cudaMemcpyDefault, r.s));
    if (o.z) PPB_CUDA(cudaMemcpyAsync(o.z, T.p_pos.as<double>() + 2 * npk, b8, cudaMemcpyDefault, r.s));
    if (o.Rf) PPB_CUDA(cudaMemcpyAsync(o.Rf, T.p_Rf.as<double>(), b8, cudaMemcpyDefault, r.s));
    if (o.FcRf) PPB_CUDA(cudaMemcpyAsync(o.FcRf, T.p_FcRf.as<float>(), b4, cudaMemcpyDefault, r.s));
    if (o.d2Rf) {
      // 0.0f0 without ioutshear (ext/CUDAExt.jl:3192)
      if (!r.want_lap) PPB_CUDA(cudaMemsetAsync(T.p_d2Rf.p, 0, b4, r.s));
      PPB_CUDA(cudaMemcpyAsync(o.d2Rf, T.p_d2Rf.as<float>(), b4, cudaMemcpyDefault, r.s));
    }
  }
  PPB_CUDA(cudaMemcpyAsync(mask, T.mask.p, N, cudaMemcpyDefault, r.s));
  PPB_CUDA(cudaStreamSynchronize(r.s));
}

void generate_fields_core(ppb_ctx* ctx, Slot& sl, const ppb_tile_params* p, float* delta, float* psi, float* psi2,
                          float* lapd) {
  PPB_REQUIRE(p->n >= 8 && p->n <= 2048, "n must be in [8, 2048]");
  PPB_REQUIRE(p->boxsize > 0, "boxsize must be positive");
  PPB_REQUIRE(p->ilpt == 1 || p->ilpt == 2, "ilpt must be 1 or 2");
  PPB_REQUIRE(ctx->sh.pk_n >= 2, "P(k) table not set (ppb_set_pk_table)");
  PPB_REQUIRE(psi2 == nullptr || p->ilpt >= 2, "psi2 needs ilpt = 2");
  PPB_REQUIRE(lapd == nullptr || p->ioutshear >= 1, "lapd needs ioutshear >= 1");
  const int n = p->n;
  const int64_t N = (int64_t)n * n * n;
  Run r{};
  r.ctx = ctx;
  r.sl = &sl;
  r.p = p;
  r.s = sl.stream;
  r.L = Launch{sl.stream, &sl.launches};
  r.plain = p->plain != 0;
  r.want_lap = p->ioutshear >= 1;
  TileRes& T = sl.tile_for(n);
  T.setup(n, r.s);
  fields_phase(r, T, n, p->boxsize);
  if (delta) copy_out(delta, T.delta.p, N * 4, r.s);
  if (psi) copy_out(psi, T.psi.p, 3 * N * 4, r.s);
  if (psi2) copy_out(psi2, T.psi2.p, 3 * N * 4, r.s);
  if (lapd) copy_out(lapd, T.lapd.p, N * 4, r.s);
  PPB_CUDA(cudaStreamSynchronize(r.s));
}

void run_tile_core(ppb_ctx* ctx, Slot& sl, const ppb_tile_params* p, const double* Rf_in, int nfilt, TileOut* o) {
  check_params(p, Rf_in, nfilt);
  PPB_REQUIRE(ctx->sh.pk_n >= 2, "P(k) table not set (ppb_set_pk_table)");
  PPB_REQUIRE(ctx->sh.has_tab, "collapse table not set (ppb_set_collapse_table)");
  const int n = p->n;
  const double box = p->boxsize;
  const int64_t N = (int64_t)n * n * n;
  Run r;
  setup_run(r, ctx, sl, p, Rf_in, nfilt, box / n);
  TileRes& T = sl.tile_for(n);
  T.setup(n, r.s);
  T.aos.ensure(pack_bytes(n));
  if (T.cap == 0) T.ensure_peaks(initial_peak_capacity(N));
  cudaEvent_t* ev = sl.stage_ev;
  PPB_CUDA(cudaEventRecord(ev[0], r.s));
  // fields and the packed gather records as one graph
  ctx->captured(sl, T.graphs, 0, n, [&] {
    fields_phase(r, T, n, box);
    launch_pack(r.L, T.aos.as<float4>(),
                FieldWindow{T.delta.as<float>(), T.psi.as<float>(), p->ilpt >= 2 ? T.psi2.as<float>() : nullptr, 0,
                            n, (int64_t)n * n, N},
                n);
  });
  PPB_CUDA(cudaEventRecord(ev[1], r.s));
  const int64_t npk = peaks_phase(r, T, n, box, {Win{0, (float)r.fcrit_val}}, n);
  PPB_CUDA(cudaEventRecord(ev[2], r.s));
  prep_phase(r, T, npk, n, 1, nullptr);
  ShellStats st{};
  shells_phase(r, T, 0, npk, n, T.aos.as<float4>(), r.want_lap ? T.lapd.as<float>() : nullptr, &st);
  PPB_CUDA(cudaEventRecord(ev[3], r.s));
  int64_t nrec = 0;
  float rmax = 0.f;
  records_phase(r, T, npk, &nrec, &rmax);
  PPB_CUDA(cudaEventRecord(ev[4], r.s));
  PPB_CUDA(cudaStreamSynchronize(r.s));
  check_shell_stats(st);
  sl.last_shell = st;
  o->nfields = p->ioutshear >= 1 ? 33 : 11;
  o->count = nrec;
  o->npeaks = npk;
  o->RTHLmax = rmax;
  o->d_records = T.rec.as<float>();
  sl.last_visits = st.visits;
  sl.last_npk = npk;
  float ms[4];
  for (int i = 0; i < 4; i++) PPB_CUDA(cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]));
  std::memcpy(sl.stage_ms, ms, sizeof(ms));
  o->device_ms = ms[0] + ms[1] + ms[2] + ms[3];
}

// run_multitile (src/MultiTile.jl:108-418): fields on the full periodic grid
// N = nsub ntile + 2 nbuff (nsub = n - 2 nbuff, alatt = boxsize / n), the
// filter bank on the full grid, peaks per tile in its nsub^3 core (tile
// (it, jt, kt) starts at cell ((it-1) nsub, (jt-1) nsub, (kt-1) nsub); on the
// lightcone with the fcrit of the tile centre's redshift and tiles beyond
// chi(z_max) dropped), and the shell analysis per tile on the tile's own
// n^3 fields.  Records are in tile order.
void run_multitile_core(ppb_ctx* ctx, Slot& sl, const ppb_tile_params* p, const double* Rf_in, int nfilt,
                        int ntile, const int32_t* tiles_in, int ntiles_in, TileOut* o) {
  check_params(p, Rf_in, nfilt);
  PPB_REQUIRE(ctx->sh.pk_n >= 2, "P(k) table not set (ppb_set_pk_table)");
  PPB_REQUIRE(ctx->sh.has_tab, "collapse table not set (ppb_set_collapse_table)");
  PPB_REQUIRE(ntile >= 1 && ntile <= 16, "ntile must be in [1, 16]");
  const int nm = p->n, nbuff = p->nbuff, nsub = nm - 2 * nbuff;
  const int64_t Ng = (int64_t)nsub * ntile + 2 * nbuff;
  PPB_REQUIRE(Ng <= 2048, "full grid nsub ntile + 2 nbuff must be <= 2048");
  const int n = (int)Ng;
  const double alatt = p->boxsize / nm, box = n * alatt, dcore = nsub * alatt;
  const int64_t N = (int64_t)n * n * n;
  Run r;
  setup_run(r, ctx, sl, p, Rf_in, nfilt, alatt);
  // tiles: the given list, else every tile in (kt, jt, it) loop order
  std::vector<std::array<int, 3>> tl;
  if (tiles_in && ntiles_in > 0) {
    for (int t = 0; t < ntiles_in; t++) {
      const int it = tiles_in[3 * t], jt = tiles_in[3 * t + 1], kt = tiles_in[3 * t + 2];
      PPB_REQUIRE(it >= 1 && it <= ntile && jt >= 1 && jt <= ntile && kt >= 1 && kt <= ntile,
                  "tile index out of range");
      tl.push_back({it, jt, kt});
    }
  } else {
    for (int kt = 1; kt <= ntile; kt++)
      for (int jt = 1; jt <= ntile; jt++)
        for (int it = 1; it <= ntile; it++) tl.push_back({it, jt, kt});
  }
  const double cen = 0.5 * (ntile + 1);
  auto centre = [&](const std::array<int, 3>& t, int d) { return (t[d] - cen) * dcore; };
  const double obs[3] = {p->cenx, p->ceny, p->cenz};
  std::vector<double> chis;
  if (p->ievol == 1) {   // lightcone: drop tiles beyond chi(z_max) (MultiTile.jl:205-216)
    const double chi_max = chi_of_z(r.Om, p->Omvac, p->h, p->z_max);
    const double half = dcore / 2.0;
    std::vector<std::array<int, 3>> keep;
    for (const auto& t : tl) {
      double d2 = 0.0;
      for (int d = 0; d < 3; d++) {
        const double e = std::max(std::fabs(centre(t, d) - obs[d]) - half, 0.0);
        d2 += e * e;
      }
      if (std::sqrt(d2) <= chi_max) keep.push_back(t);
    }
    tl.swap(keep);
    chis = ctx->chi_table(r.Om, p->Omvac, p->h, p->z_max + 1.0);
  }
  const int nwin = (int)tl.size();
  std::vector<Win> wins(nwin);
  std::vector<double> tcen(3 * std::max(nwin, 1), 0.0);
  for (int t = 0; t < nwin; t++) {
    const int64_t i1 = (int64_t)(tl[t][0] - 1) * nsub, j1 = (int64_t)(tl[t][1] - 1) * nsub,
                  k1 = (int64_t)(tl[t][2] - 1) * nsub;
    wins[t].off = i1 + (int64_t)n * j1 + (int64_t)n * n * k1;
    for (int d = 0; d < 3; d++) tcen[3 * t + d] = centre(tl[t], d);
    double fc = r.fcrit_val;
    if (p->ievol == 1) {   // fcrit at the tile centre's redshift (MultiTile.jl:238-243)
      double d2 = 0.0;
      for (int d = 0; d < 3; d++) d2 += (tcen[3 * t + d] - obs[d]) * (tcen[3 * t + d] - obs[d]);
      fc = fsc_of_z(*r.G, chi_to_z_host(chis, p->z_max + 1.0, std::sqrt(d2)));
    }
    wins[t].fcrit = (float)fc;
  }
  TileRes& T = sl.tile_for(n);
  T.setup(n, r.s);
  if (T.cap == 0) T.ensure_peaks(initial_peak_capacity(N));
  sl.tcen.ensure(tcen.size() * 8);
  PPB_CUDA(cudaMemcpyAsync(sl.tcen.p, tcen.data(), tcen.size() * 8, cudaMemcpyHostToDevice, r.s));
  cudaEvent_t* ev = sl.stage_ev;
  PPB_CUDA(cudaEventRecord(ev[0], r.s));
  ctx->captured(sl, T.graphs, 0, n, [&] { fields_phase(r, T, n, box); });
  PPB_CUDA(cudaEventRecord(ev[1], r.s));
  int64_t npk = 0;
  if (nwin > 0) npk = peaks_phase(r, T, n, box, wins, nm);
  PPB_CUDA(cudaEventRecord(ev[2], r.s));
  prep_phase(r, T, npk, nm, nwin, sl.tcen.as<double>());
  // peaks per tile (the sorted list is grouped by tile)
  std::vector<int> cnt(std::max(nwin, 1), 0);
  if (npk > 0) {
    int tbits = 0;
    while ((1 << tbits) < nwin) tbits++;
    PPB_CUDA(cudaMemsetAsync(T.count.p, 0, 64, r.s));
    sl.tcount.ensure(cnt.size() * 4);
    PPB_CUDA(cudaMemsetAsync(sl.tcount.p, 0, cnt.size() * 4, r.s));
    tile_count_kernel<<<(unsigned)((npk + 255) / 256), 256, 0, r.s>>>(T.keys_s.as<unsigned long long>(), (int)npk,
                                                                      40 + r.fbits, sl.tcount.as<int>());
    PPB_LAUNCHED(sl.launches);
    PPB_CUDA(cudaMemcpyAsync(cnt.data(), sl.tcount.p, cnt.size() * 4, cudaMemcpyDeviceToHost, r.s));
    PPB_CUDA(cudaStreamSynchronize(r.s));
  }
  // shells per tile on the tile's own fields (MultiTile.jl:286-327)
  const int64_t Nt = (int64_t)nm * nm * nm;
  ShellStats st{};
  int64_t p0 = 0;
  for (int t = 0; t < nwin; t++) {
    const int64_t p1 = p0 + cnt[t];
    if (p1 > p0) {
      // the tile's chain: its packed records and Laplacian window, then the
      // shell stage, captured together as one graph per sub-batch
      sl.t_aos.ensure(pack_bytes(nm));
      if (r.want_lap) sl.t_lapd.ensure(Nt * 4);
      const float* lapd = r.want_lap ? sl.t_lapd.as<float>() : nullptr;
      const int64_t off = wins[t].off;
      shells_phase(r, T, p0, p1, nm, sl.t_aos.as<float4>(), lapd, &st, [&] {
        launch_pack(r.L, sl.t_aos.as<float4>(),
                    FieldWindow{T.delta.as<float>(), T.psi.as<float>(), p->ilpt >= 2 ? T.psi2.as<float>() : nullptr,
                                off, n, (int64_t)n * n, N},
                    nm);
        if (r.want_lap)
          launch_extract(r.L, sl.t_lapd.as<float>(), T.lapd.as<float>(), off, n, (int64_t)n * n, nm);
      });
    }
    p0 = p1;
  }
  PPB_CUDA(cudaEventRecord(ev[3], r.s));
  int64_t nrec = 0;
  float rmax = 0.f;
  records_phase(r, T, npk, &nrec, &rmax);
  PPB_CUDA(cudaEventRecord(ev[4], r.s));
  PPB_CUDA(cudaStreamSynchronize(r.s));
  check_shell_stats(st);
  sl.last_shell = st;
  o->nfields = p->ioutshear >= 1 ? 33 : 11;
  o->count = nrec;
  o->npeaks = npk;
  o->RTHLmax = rmax;
  o->d_records = T.rec.as<float>();
  sl.last_visits = st.visits;
  sl.last_npk = npk;
  float ms[4];
  for (int i = 0; i < 4; i++) PPB_CUDA(cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]));
  std::memcpy(sl.stage_ms, ms, sizeof(ms));
  o->device_ms = ms[0] + ms[1] + ms[2] + ms[3];
}

// the coarse grid of run_multitile_split (src/MultiResolution.jl:592-612):
// coarse_grid, else ntile coarse_factor, else the divisor m of N (2 <= m <=
// N/2) whose block N/m is closest to nmesh/3 (the first such m)
int split_coarse_grid(int64_t N, int nmesh, int ntile, int coarse_factor, int coarse_grid) {
  if (coarse_grid > 0) return coarse_grid;
  if (coarse_factor > 0) return ntile * coarse_factor;
  const int64_t target = nmesh / 3;
  int64_t best = 0, best_dist = N;
  for (int64_t m = 2; m <= N / 2; m++) {
    if (N % m != 0) continue;
    const int64_t dist = std::llabs(N / m - target);
    if (dist < best_dist) {
      best_dist = dist;
      best = m;
    }
  }
  return (int)best;
}

namespace {

// dst (device, `used` bytes kept) grown to hold `more` bytes beyond used
void grow_keep(DevBuf& dst, size_t used, size_t more, cudaStream_t s) {
  if (used + more <= dst.bytes) return;
  const size_t nb = std::max(used + more, 2 * dst.bytes);
  void* np = nullptr;
  PPB_CUDA(cudaMalloc(&np, nb));
  if (used) PPB_CUDA(cudaMemcpyAsync(np, dst.p, used, cudaMemcpyDeviceToDevice, s));
  PPB_CUDA(cudaStreamSynchronize(s));
  dst.release();
  dst.p = np;
  dst.bytes = nb;
}

}  // namespace

// run_multitile_split (src/MultiResolution.jl:523-1236) with use_gpu: the
// coarse noise and coarse delta / psi on M^3 once, then per tile the fields
// by the split (isolated convolution of the Hoffman-Ribak residual plus the
// tricubic coarse field; tile-local 2LPT and Laplacian), the filter bank and
// peak search on the tile's own nmesh^3 grid (fcrit of the tile centre on
// the lightcone), the shell analysis and the records, in tile order.
void run_multitile_split_core(ppb_ctx* ctx, Slot& sl, const ppb_tile_params* p, const double* Rf_in, int nfilt,
                              int ntile, int coarse_factor, int coarse_grid, const int32_t* tiles_in, int ntiles_in,
                              TileOut* o) {
  check_params(p, Rf_in, nfilt);
  PPB_REQUIRE(ctx->sh.pk_n >= 2, "P(k) table not set (ppb_set_pk_table)");
  PPB_REQUIRE(ctx->sh.has_tab, "collapse table not set (ppb_set_collapse_table)");
  PPB_REQUIRE(ntile >= 1 && ntile <= 64, "ntile must be in [1, 64]");
  const int nm = p->n, nbuff = p->nbuff, nsub = nm - 2 * nbuff;
  PPB_REQUIRE(nm <= 640, "nmesh must be <= 640 (isolated convolution box (2 nmesh)^3)");
  const int64_t N = (int64_t)nsub * ntile + 2 * nbuff;
  const int M = split_coarse_grid(N, nm, ntile, coarse_factor, coarse_grid);
  PPB_REQUIRE(M >= 1 && N % M == 0, "N = nsub ntile + 2 nbuff must be divisible by the coarse grid M");
  PPB_REQUIRE(N / M <= 1024 && M <= 1024 && N <= (1 << 20), "coarse grid out of range");
  const double alatt = p->boxsize / nm, box_full = (double)N * alatt, box_local = nm * alatt, dcore = nsub * alatt;
  const int64_t Nt = (int64_t)nm * nm * nm;
  Run r;
  setup_run(r, ctx, sl, p, Rf_in, nfilt, alatt);
  // tiles: the given list, else every tile in (kt, jt, it) loop order
  std::vector<std::array<int, 3>> tl;
  if (tiles_in && ntiles_in > 0) {
    for (int t = 0; t < ntiles_in; t++) {
      const int it = tiles_in[3 * t], jt = tiles_in[3 * t + 1], kt = tiles_in[3 * t + 2];
      PPB_REQUIRE(it >= 1 && it <= ntile && jt >= 1 && jt <= ntile && kt >= 1 && kt <= ntile,
                  "tile index out of range");
      tl.push_back({it, jt, kt});
    }
  } else {
    for (int kt = 1; kt <= ntile; kt++)
      for (int jt = 1; jt <= ntile; jt++)
        for (int it = 1; it <= ntile; it++) tl.push_back({it, jt, kt});
  }
  const double cen = 0.5 * (ntile + 1);
  auto centre = [&](const std::array<int, 3>& t, int d) { return (t[d] - cen) * dcore; };
  const double obs[3] = {p->cenx, p->ceny, p->cenz};
  std::vector<double> chis;
  if (p->ievol == 1) {   // lightcone: drop tiles beyond chi(z_max) (:680-692)
    const double chi_max = chi_of_z(r.Om, p->Omvac, p->h, p->z_max);
    const double half = dcore / 2.0;
    std::vector<std::array<int, 3>> keep;
    for (const auto& t : tl) {
      double d2 = 0.0;
      for (int d = 0; d < 3; d++) {
        const double e = std::max(std::fabs(centre(t, d) - obs[d]) - half, 0.0);
        d2 += e * e;
      }
      if (std::sqrt(d2) <= chi_max) keep.push_back(t);
    }
    tl.swap(keep);
    chis = ctx->chi_table(r.Om, p->Omvac, p->h, p->z_max + 1.0);
  }
  const int nt = (int)tl.size();
  std::vector<double> tcen(3 * std::max(nt, 1), 0.0);
  std::vector<float> fcrit_t(std::max(nt, 1), (float)r.fcrit_val);
  for (int t = 0; t < nt; t++) {
    for (int d = 0; d < 3; d++) tcen[3 * t + d] = centre(tl[t], d);
    if (p->ievol == 1) {   // fcrit at the tile centre's redshift (:864-871)
      double d2 = 0.0;
      for (int d = 0; d < 3; d++) d2 += (tcen[3 * t + d] - obs[d]) * (tcen[3 * t + d] - obs[d]);
      fcrit_t[t] = (float)fsc_of_z(*r.G, chi_to_z_host(chis, p->z_max + 1.0, std::sqrt(d2)));
    }
  }
  sl.tcen.ensure(tcen.size() * 8);
  PPB_CUDA(cudaMemcpyAsync(sl.tcen.p, tcen.data(), tcen.size() * 8, cudaMemcpyHostToDevice, r.s));
  // phase 0 / 1a: coarse noise, coarse delta and psi (:596-632; the coarse
  // 2LPT and Laplacian of :635-667 are never read afterwards)
  const int64_t Mc = (int64_t)M * M * M, fs = (Mc + 3) & ~(int64_t)3;
  sl.mr_in.ensure(Mc * 4);
  sl.mr_aux.ensure(4 * fs * 4 + Mc * 16);
  float* cnoise = sl.mr_in.as<float>();
  float* cf = sl.mr_aux.as<float>();
  float4* cf4 = reinterpret_cast<float4*>(cf + 4 * fs);   // 16-byte aligned: fs is a multiple of 4
  cudaEvent_t* ev = sl.stage_ev;
  PPB_CUDA(cudaEventRecord(ev[0], r.s));
  launch_coarse_noise(r.L, cnoise, N, M, p->seed);
  mr_coarse_device(ctx, sl, cnoise, M, box_full, 1, 0, cf, fs);
  launch_interleave4(r.L, cf4, cf, fs, Mc);
  TileRes& T = sl.tile_for(nm);
  T.setup(nm, r.s);
  T.aos.ensure(pack_bytes(nm));
  if (T.cap == 0) T.ensure_peaks(initial_peak_capacity(Nt));
  const int nf = p->ioutshear >= 1 ? 33 : 11;
  size_t used = 0;
  int64_t nrec_tot = 0, npk_tot = 0;
  float rmax_tot = 0.f;
  float ms[4] = {0.f, 0.f, 0.f, 0.f};
  ShellStats st{};
  PPB_CUDA(cudaEventRecord(ev[1], r.s));
  PPB_CUDA(cudaEventSynchronize(ev[1]));
  PPB_CUDA(cudaEventElapsedTime(&ms[0], ev[0], ev[1]));
  for (int t = 0; t < nt; t++) {
    const int64_t i0 = (int64_t)(tl[t][0] - 1) * nsub - nbuff, j0 = (int64_t)(tl[t][1] - 1) * nsub - nbuff,
                  k0 = (int64_t)(tl[t][2] - 1) * nsub - nbuff;
    PPB_CUDA(cudaEventRecord(ev[0], r.s));
    // fields (:728-847)
    mr_split_tile_fields(ctx, sl, T, cnoise, reinterpret_cast<const float*>(cf4), M, N, i0, j0, k0, nm, box_local,
                         p->seed);
    mr_tile_2lpt_lap(ctx, sl, T, nm, box_local, p->ilpt >= 2 ? T.psi2.as<float>() : nullptr,
                     r.want_lap ? T.lapd.as<float>() : nullptr);
    launch_hermitise(r.L, T.dk.as<float2>(), nm, 1);
    launch_pack(r.L, T.aos.as<float4>(),
                FieldWindow{T.delta.as<float>(), T.psi.as<float>(), p->ilpt >= 2 ? T.psi2.as<float>() : nullptr, 0,
                            nm, (int64_t)nm * nm, Nt},
                nm);
    PPB_CUDA(cudaEventRecord(ev[1], r.s));
    // peaks on the tile's grid (:856-906), shells (:908-1021), records
    const int64_t npk = peaks_phase(r, T, nm, box_local, {Win{0, fcrit_t[t]}}, nm);
    PPB_CUDA(cudaEventRecord(ev[2], r.s));
    prep_phase(r, T, npk, nm, 1, sl.tcen.as<double>() + 3 * t);
    shells_phase(r, T, 0, npk, nm, T.aos.as<float4>(), r.want_lap ? T.lapd.as<float>() : nullptr, &st);
    PPB_CUDA(cudaEventRecord(ev[3], r.s));
    int64_t nrec = 0;
    float rmax = 0.f;
    records_phase(r, T, npk, &nrec, &rmax);
    if (nrec > 0) {
      const size_t bytes = (size_t)nrec * nf * 4;
      grow_keep(sl.mr_rec, used, bytes, r.s);
      PPB_CUDA(cudaMemcpyAsync((char*)sl.mr_rec.p + used, T.rec.p, bytes, cudaMemcpyDeviceToDevice, r.s));
      used += bytes;
    }
    PPB_CUDA(cudaEventRecord(ev[4], r.s));
    PPB_CUDA(cudaEventSynchronize(ev[4]));
    float e[4];
    for (int i = 0; i < 4; i++) PPB_CUDA(cudaEventElapsedTime(&e[i], ev[i], ev[i + 1]));
    ms[0] += e[0];
    ms[1] += e[1];
    ms[2] += e[2];
    ms[3] += e[3];
    nrec_tot += nrec;
    npk_tot += npk;
    rmax_tot = std::max(rmax_tot, rmax);
  }
  check_shell_stats(st);
  sl.last_shell = st;
  o->nfields = nf;
  o->count = nrec_tot;
  o->npeaks = npk_tot;
  o->RTHLmax = nrec_tot > 0 ? rmax_tot : 0.f;
  o->d_records = sl.mr_rec.as<float>();
  sl.last_visits = st.visits;
  sl.last_npk = npk_tot;
  std::memcpy(sl.stage_ms, ms, sizeof(ms));
  o->device_ms = ms[0] + ms[1] + ms[2] + ms[3];
}

}  // namespace ppb
