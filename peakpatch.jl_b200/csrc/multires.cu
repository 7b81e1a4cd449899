// multires.cu — C-ABI entry points of the multi-resolution (MUSIC-style)
// tile fields of run_multitile_split (src/MultiResolution.jl), the drop-in
// for the reference's GPU plug-in functions isolated_convolve_gpu(_multi),
// interpolate_to_tile_gpu, compute_2lpt_gpu and compute_laplacian_gpu
// (stubs src/PeakPatch.jl:255-339) and for the CPU steps around them
// (_downsample_noise, _generate_extended_residual, the coarse phase).
//
// All of them run on the context's synchronous slot; buffers stay resident
// between calls (the isolated convolution keeps its plans for the last padded
// size, the periodic kernels use the slot's per-size tile buffers).
#include <algorithm>
#include <cmath>
#include <vector>

#include "ppb_ctx.h"

using namespace ppb;

namespace ppb {

// ---------------------------------------------------------------------------
// isolated-convolution resources
// ---------------------------------------------------------------------------
// the pruned transforms of a zero-padded box: 2-D (y, x) real<->complex
// transforms over `planes` consecutive z-planes, and the 1-D complex
// transform along z of every (y, x) column, all in place
static cufftHandle plan_planes(int n, cufftType t, int planes, size_t* ws) {
  cufftHandle h;
  PPB_CUFFT(cufftCreate(&h));
  PPB_CUFFT(cufftSetAutoAllocation(h, 0));
  long long dims[2] = {n, n};
  const long long nh = n / 2 + 1;
  long long cemb[2] = {n, nh}, remb[2] = {n, 2 * nh};
  const long long cdist = (long long)n * nh, rdist = 2 * cdist;
  if (t == CUFFT_R2C)
    PPB_CUFFT(cufftMakePlanMany64(h, 2, dims, remb, 1, rdist, cemb, 1, cdist, t, planes, ws));
  else
    PPB_CUFFT(cufftMakePlanMany64(h, 2, dims, cemb, 1, cdist, remb, 1, rdist, t, planes, ws));
  return h;
}

static cufftHandle plan_columns(int n, size_t* ws) {
  cufftHandle h;
  PPB_CUFFT(cufftCreate(&h));
  PPB_CUFFT(cufftSetAutoAllocation(h, 0));
  long long dims[1] = {n};
  const long long plane = (long long)n * (n / 2 + 1);
  long long emb[1] = {n};
  PPB_CUFFT(cufftMakePlanMany64(h, 1, dims, emb, plane, 1, emb, plane, 1, CUFFT_C2C, plane, ws));
  return h;
}

IsoRes::~IsoRes() {
  for (cufftHandle h : {f2d, i2d, col})
    if (h) cufftDestroy(h);
}

void IsoRes::setup(int nn, int nb, cudaStream_t s) {
  const int64_t modes = (int64_t)(nn / 2 + 1) * nn * nn;
  if (nn != n2) {
    for (cufftHandle* h : {&f2d, &i2d, &col})
      if (*h) { cufftDestroy(*h); *h = 0; }
    n2 = 0;
    size_t w[3] = {0, 0, 0};
    f2d = plan_planes(nn, CUFFT_R2C, nn / 2, &w[0]);
    i2d = plan_planes(nn, CUFFT_C2R, nn / 2, &w[1]);
    col = plan_columns(nn, &w[2]);
    ws.ensure(std::max<size_t>(std::max(w[0], std::max(w[1], w[2])), 256));
    for (cufftHandle h : {f2d, i2d, col}) PPB_CUFFT(cufftSetWorkArea(h, ws.p));
    spec.ensure(modes * 8);
    amp.ensure(amp_table_size(nn) * 8);
    amp_box = 0.0;
    n2 = nn;
  }
  for (cufftHandle h : {f2d, i2d, col}) PPB_CUFFT(cufftSetStream(h, s));
  work.ensure((size_t)nb * modes * 8);
  batch = (int)(work.bytes / ((size_t)modes * 8));
}

// forward transform of the zero-padded box in spec (input nonzero on planes
// z < n2/2 only): the 2-D transform of those planes, then every z-column
static void iso_forward(Slot& sl, IsoRes& iso) {
  PPB_CUFFT(cufftExecR2C(iso.f2d, iso.spec.as<float>(), iso.spec.as<cufftComplex>()));
  PPB_CUFFT(cufftExecC2C(iso.col, iso.spec.as<cufftComplex>(), iso.spec.as<cufftComplex>(), CUFFT_FORWARD));
  sl.launches += 2;
}

// inverse transform of the half-spectrum at w, valid on the z-planes
// [z0, z0 + nz): every z-column, then the 2-D transform of n2/2 planes that
// cover them (of all planes when nz > n2/2)
static void iso_inverse(Slot& sl, IsoRes& iso, float2* w, int z0, int nz) {
  const int half = iso.n2 / 2;
  const int64_t plane = (int64_t)iso.n2 * (half + 1);
  cufftComplex* c = reinterpret_cast<cufftComplex*>(w);
  PPB_CUFFT(cufftExecC2C(iso.col, c, c, CUFFT_INVERSE));
  sl.launches++;
  const int starts[2] = {nz > half ? 0 : std::min(z0, iso.n2 - half), half};
  for (int h = 0; h < (nz > half ? 2 : 1); h++) {
    cufftComplex* p = c + starts[h] * plane;
    PPB_CUFFT(cufftExecC2R(iso.i2d, p, reinterpret_cast<float*>(p)));
    sl.launches++;
  }
}

// the amplitude table of the padded box of side `box` (rebuilt when the box
// or the P(k) table changed)
static const double* iso_amp(ppb_ctx* ctx, Slot& sl, IsoRes& iso, double box) {
  if (iso.amp_box != box || iso.amp_pk != ctx->sh.pk_version) {
    const double post = 1.0 / ((double)iso.n2 * (double)iso.n2 * (double)iso.n2);
    launch_amp_table(Launch{sl.stream, &sl.launches}, iso.amp.as<double>(), iso.n2, box, ctx->sh.pk_lk.as<double>(),
                     ctx->sh.pk_lp.as<double>(), ctx->sh.pk_n, post);
    iso.amp_box = box;
    iso.amp_pk = ctx->sh.pk_version;
  }
  return iso.amp.as<double>();
}


// ---------------------------------------------------------------------------
// device-level stages (shared by the entry points below and the split driver)
// ---------------------------------------------------------------------------
void mr_isolated_device(ppb_ctx* ctx, Slot& sl, const float* d_noise, int n_input, double boxsize_local, int n,
                        const int32_t* kernels, int nk, int nshell, float* const* outs) {
  cudaStream_t s = sl.stream;
  Launch L{s, &sl.launches};
  const int n2 = 2 * n_input, nh2 = n2 / 2 + 1;
  const int64_t modes = (int64_t)nh2 * n2 * n2, px = 2 * (int64_t)nh2;
  // kernels per transfer pass: all of them (up to 4) unless memory is short
  int batch = std::min(nk, 4);
  if (!sl.iso) sl.iso.reset(new IsoRes());
  IsoRes& iso = *sl.iso;
  if (iso.n2 != n2 || iso.batch < batch) {
    size_t fr = 0, tot = 0;
    PPB_CUDA(cudaMemGetInfo(&fr, &tot));
    const size_t have = fr + iso.work.bytes + iso.spec.bytes;
    while (batch > 1 && (size_t)(batch + 2) * modes * 8 > have) batch--;
  }
  iso.setup(n2, batch, s);
  batch = std::min(iso.batch, std::min(nk, kMaxKSpecs));
  launch_pad(L, d_noise, iso.spec.as<float>(), n_input, n2, px);
  iso_forward(sl, iso);
  // dx = boxsize_local / n; the padded box is n2 * dx (src/MultiResolution.jl:249-259)
  const double box = (double)n2 * (boxsize_local / (double)n);
  const double post = 1.0 / ((double)n2 * (double)n2 * (double)n2);
  const double* amp = iso_amp(ctx, sl, iso, box);
  for (int b0 = 0; b0 < nk; b0 += batch) {
    const int g = std::min(batch, nk - b0);
    int kind[kMaxKSpecs], d1[kMaxKSpecs], d2[kMaxKSpecs];
    for (int q = 0; q < g; q++) {
      kind[q] = kernels[3 * (b0 + q)];
      d1[q] = kernels[3 * (b0 + q) + 1];
      d2[q] = kernels[3 * (b0 + q) + 2];
    }
    launch_kspace(L, amp, iso.spec.as<float2>(), iso.work.as<float2>(), modes, n2, box, kind, d1, d2, g, post);
    for (int q = 0; q < g; q++) {
      float2* w = iso.work.as<float2>() + q * modes;
      iso_inverse(sl, iso, w, nshell, n);
      launch_extract(L, outs[b0 + q], reinterpret_cast<const float*>(w), (int64_t)nshell * (1 + px + px * n2), px,
                     px * n2, n);
    }
  }
}

void mr_tile_2lpt_lap(ppb_ctx* ctx, Slot& sl, TileRes& T, int n, double box, float* psi2, float* lapd) {
  (void)ctx;
  Launch L{sl.stream, &sl.launches};
  const int64_t N = (int64_t)n * n * n, Mk = (int64_t)(n / 2 + 1) * n * n;
  const double post = 1.0 / ((double)n * (double)n * (double)n);
  auto forward = [&](float* src) {
    PPB_CUFFT(cufftExecR2C(T.r2c, src, T.dk.as<cufftComplex>()));
    sl.launches++;
  };
  forward(T.delta.as<float>());
  if (psi2) {
    // phi_11, phi_22, phi_33, phi_12, phi_13, phi_23 (:812-821)
    const int pk6[6] = {3, 3, 3, 3, 3, 3}, pa[6] = {1, 2, 3, 1, 1, 2}, pb[6] = {1, 2, 3, 2, 3, 3};
    launch_kspace(L, nullptr, T.dk.as<float2>(), T.kw.as<float2>(), Mk, n, box, pk6, pa, pb, 6, post);
    PPB_CUFFT(cufftExecC2R(T.c2r6, T.kw.as<cufftComplex>(), T.rw.as<float>()));
    sl.launches++;
    launch_src2_trace(L, T.delta.as<float>(), T.rw.as<float>(), T.rw.as<float>(), n, n, (int64_t)n * n, N);
    // rfft(src2) into the first phi slot (its transform has consumed it), so
    // T.dk keeps rfft(delta)
    PPB_CUFFT(cufftExecR2C(T.r2c, T.rw.as<float>(), T.kw.as<cufftComplex>()));
    sl.launches++;
    const int k2[3] = {2, 2, 2}, da[3] = {1, 2, 3}, db[3] = {0, 0, 0};
    launch_kspace(L, nullptr, T.kw.as<float2>(), T.kw.as<float2>() + Mk, Mk, n, box, k2, da, db, 3, post);
    PPB_CUFFT(cufftExecC2R(T.c2r3, T.kw.as<cufftComplex>() + Mk, psi2));
    sl.launches++;
  }
  if (lapd) {
    const int k4[1] = {4}, z[1] = {0};
    launch_kspace(L, nullptr, T.dk.as<float2>(), T.kw.as<float2>(), Mk, n, box, k4, z, z, 1, post);
    PPB_CUFFT(cufftExecC2R(T.c2r1, T.kw.as<cufftComplex>(), lapd));
    sl.launches++;
  }
}

void mr_split_tile_fields(ppb_ctx* ctx, Slot& sl, TileRes& T, const float* cnoise, const float* cf4, int M, int64_t N,
                          int64_t i0, int64_t j0, int64_t k0, int nm, double box_local, uint64_t seed) {
  cudaStream_t s = sl.stream;
  Launch L{s, &sl.launches};
  const int n2 = 2 * nm, nh2 = n2 / 2 + 1;
  const int64_t modes = (int64_t)nh2 * n2 * n2, px = 2 * (int64_t)nh2, Nt = (int64_t)nm * nm * nm;
  if (!sl.iso) sl.iso.reset(new IsoRes());
  IsoRes& iso = *sl.iso;
  iso.setup(n2, 4, s);
  // the residual written straight into the zero-padded box (:731-733, 254-255)
  PPB_CUDA(cudaMemsetAsync(iso.spec.p, 0, (size_t)modes * 8, s));
  launch_residual(L, cnoise, iso.spec.as<float>(), M, N, i0, j0, k0, nm, seed, px, px * n2);
  iso_forward(sl, iso);
  // delta, psi_x, psi_y, psi_z of the isolated convolution (:740-752)
  const double box = (double)n2 * (box_local / (double)nm);
  const int kind[4] = {0, 1, 1, 1}, d1[4] = {0, 1, 2, 3}, d2[4] = {0, 0, 0, 0};
  launch_kspace(L, iso_amp(ctx, sl, iso, box), iso.spec.as<float2>(), iso.work.as<float2>(), modes, n2, box, kind, d1,
                d2, 4, 1.0 / ((double)n2 * (double)n2 * (double)n2));
  for (int q = 0; q < 4; q++) iso_inverse(sl, iso, iso.work.as<float2>() + q * modes, 0, nm);
  // plus the tricubic coarse fields, read from the transforms in place
  // (:764-795): one pass writes the four tile fields
  sl.mr_axis.ensure((size_t)3 * nm * 32);
  int4* aidx = sl.mr_axis.as<int4>();
  float4* awt = reinterpret_cast<float4*>(aidx + 3 * nm);
  launch_axis_weights(L, aidx, awt, M, N, i0, j0, k0, nm);
  float* out[4] = {T.delta.as<float>(), T.psi.as<float>(), T.psi.as<float>() + Nt, T.psi.as<float>() + 2 * Nt};
  const float* w = iso.work.as<float>();
  const float* base[4] = {w, w + 2 * modes, w + 4 * modes, w + 6 * modes};
  launch_tricubic(L, aidx, awt, M, nm, 4, cf4, out, base, 0, px, px * n2);
}

void mr_coarse_device(ppb_ctx* ctx, Slot& sl, const float* d_noise, int M, double boxsize_full, int ilpt,
                      int ioutshear, float* o, int64_t fs) {
  const double* lk = ctx->sh.pk_lk.as<double>();
  const double* lp = ctx->sh.pk_lp.as<double>();
  const int np = ctx->sh.pk_n;
  Launch L{sl.stream, &sl.launches};
  const int64_t N = (int64_t)M * M * M, Mk = (int64_t)(M / 2 + 1) * M * M;
  TileRes& tr = sl.tile_for(M);
  tr.setup(M, sl.stream);
  PPB_CUDA(cudaMemcpyAsync(tr.delta.p, d_noise, N * 4, cudaMemcpyDeviceToDevice, sl.stream));
  PPB_CUFFT(cufftExecR2C(tr.r2c, tr.delta.as<float>(), tr.dk.as<cufftComplex>()));
  sl.launches++;
  const double post = 1.0 / ((double)M * (double)M * (double)M);
  sl.mr_amp.ensure(amp_table_size(M) * 8);
  const double* amp = sl.mr_amp.as<double>();
  launch_amp_table(L, sl.mr_amp.as<double>(), M, boxsize_full, lk, lp, np, post);
  auto c2r_into = [&](int q, float* dst) {
    PPB_CUFFT(cufftExecC2R(tr.c2r1, tr.kw.as<cufftComplex>() + q * Mk, dst));
    sl.launches++;
  };
  {  // delta and psi_d (:621-632), lapd (:662-667)
    int kind[5] = {0, 1, 1, 1, 4}, a[5] = {0, 1, 2, 3, 0}, b[5] = {0, 0, 0, 0, 0};
    const int g = ioutshear >= 1 ? 5 : 4;
    launch_kspace(L, amp, tr.dk.as<float2>(), tr.kw.as<float2>(), Mk, M, boxsize_full, kind, a, b, g, post);
    for (int q = 0; q < 4; q++) c2r_into(q, o + q * fs);
    if (g == 5) c2r_into(4, o + 7 * fs);
  }
  if (ilpt >= 2) {  // the 2LPT source and displacements (:635-659)
    const int pk6[6] = {3, 3, 3, 3, 3, 3}, pa[6] = {1, 2, 3, 1, 1, 2}, pb[6] = {1, 2, 3, 2, 3, 3};
    launch_kspace(L, amp, tr.dk.as<float2>(), tr.kw.as<float2>(), Mk, M, boxsize_full, pk6, pa, pb, 6, post);
    PPB_CUFFT(cufftExecC2R(tr.c2r6, tr.kw.as<cufftComplex>(), tr.rw.as<float>()));
    sl.launches++;
    launch_src2_trace(L, o, tr.rw.as<float>(), tr.rw.as<float>(), M, M, (int64_t)M * M, N);
    PPB_CUFFT(cufftExecR2C(tr.r2c, tr.rw.as<float>(), tr.dk.as<cufftComplex>()));
    sl.launches++;
    const int k2[3] = {2, 2, 2}, da[3] = {1, 2, 3}, db[3] = {0, 0, 0};
    launch_kspace(L, amp, tr.dk.as<float2>(), tr.kw.as<float2>(), Mk, M, boxsize_full, k2, da, db, 3, post);
    for (int q = 0; q < 3; q++) c2r_into(q, o + (4 + q) * fs);
  }
}

}  // namespace ppb

namespace {

// the reference's frequency kernels (kernel_fn_id, dim1, dim2) accepted by
// isolated_convolve_gpu (src/PeakPatch.jl:261-272)
void check_kernel(int kind, int d1, int d2) {
  PPB_REQUIRE(kind >= 0 && kind <= 4, "kernel_fn_id must be 0..4");
  if (kind == 1 || kind == 2 || kind == 3) PPB_REQUIRE(d1 >= 1 && d1 <= 3, "dim1 must be 1..3");
  if (kind == 3) PPB_REQUIRE(d2 >= 1 && d2 <= 3, "dim2 must be 1..3");
}

void check_coarse(int64_t N, int M) {
  PPB_REQUIRE(N >= 1 && M >= 1 && N % M == 0, "N must be a positive multiple of M");
  PPB_REQUIRE(N / M <= 1024, "block N/M above 1024");
  PPB_REQUIRE(N <= (1ll << 20), "N above 2^20");
  PPB_REQUIRE((int64_t)M * M * M <= (1ll << 30), "M^3 above 2^30");
}

void check_tile(int it, int jt, int kt, int nsub, int nmesh) {
  PPB_REQUIRE(it >= 1 && jt >= 1 && kt >= 1, "tile numbers are 1-based");
  PPB_REQUIRE(nmesh >= 1 && nsub >= 1 && nsub <= nmesh, "need 1 <= nsub <= nmesh");
  PPB_REQUIRE(nmesh <= 2048, "nmesh above 2048");
}

// 0-based global origin of a tile's region extended by `ext` cells
// (src/MultiResolution.jl:207-209, 1-based there)
int64_t origin(int t, int nsub, int nmesh, int ext) { return (int64_t)(t - 1) * nsub - (nmesh - nsub) / 2 - ext; }

template <class F>
int32_t guarded(ppb_ctx* ctx, F&& body) {
  if (!ctx) return PPB_ERR_INVALID;
  std::lock_guard<std::recursive_mutex> lk(ctx->mu);
  try {
    PPB_CUDA(cudaSetDevice(ctx->device));
    body();
    return PPB_OK;
  } catch (const ppb::Error& e) {
    ctx->set_error(e.msg);
    return e.code;
  } catch (...) {
    ctx->set_error("unknown error");
    return PPB_ERR_INVALID;
  }
}

// device buffer for a result of `bytes`: the caller's own when it is device
// memory, else the staging buffer (copied out by finish_out)
float* out_buffer(float* dst, DevBuf& stage, size_t bytes) {
  if (is_device_ptr(dst)) return dst;
  stage.ensure(bytes);
  return stage.as<float>();
}

void finish_out(float* dst, const float* dev, size_t bytes, cudaStream_t s) {
  if (dst != dev) PPB_CUDA(cudaMemcpyAsync(dst, dev, bytes, cudaMemcpyDeviceToHost, s));
}

// the caller's field copied into the slot's tile buffers of size n
TileRes& periodic_setup(ppb_ctx* ctx, const float* delta_tile, int n) {
  Slot& sl = ctx->sync;
  TileRes& tr = sl.tile_for(n);
  tr.setup(n, sl.stream);
  const int64_t N = (int64_t)n * n * n;
  PPB_CUDA(cudaMemcpyAsync(tr.delta.p, delta_tile, N * 4, cudaMemcpyDefault, sl.stream));
  return tr;
}

}  // namespace

extern "C" {

int32_t ppb_downsample_noise(ppb_ctx* ctx, int64_t N, int32_t M, uint64_t seed, float* out) {
  return guarded(ctx, [&] {
    PPB_REQUIRE(out, "null argument");
    check_coarse(N, M);
    Slot& sl = ctx->sync;
    const size_t bytes = (size_t)M * M * M * 4;
    float* d = out_buffer(out, sl.mr_out, bytes);
    launch_coarse_noise(Launch{sl.stream, &sl.launches}, d, N, M, seed);
    finish_out(out, d, bytes, sl.stream);
    PPB_CUDA(cudaStreamSynchronize(sl.stream));
  });
}

int32_t ppb_extended_residual(ppb_ctx* ctx, const float* coarse, int32_t M, int32_t it, int32_t jt, int32_t kt,
                              int32_t nsub, int32_t nmesh, int64_t N, uint64_t seed, int32_t nshell, float* out) {
  return guarded(ctx, [&] {
    PPB_REQUIRE(coarse && out, "null argument");
    check_coarse(N, M);
    check_tile(it, jt, kt, nsub, nmesh);
    PPB_REQUIRE(nshell >= 0 && nmesh + 2 * (int64_t)nshell <= 4096, "nshell out of range");
    Slot& sl = ctx->sync;
    const int next = nmesh + 2 * nshell;
    const size_t bytes = (size_t)next * next * next * 4;
    const float* c = (const float*)stage_in(sl.mr_in, coarse, (size_t)M * M * M * 4, sl.stream);
    float* d = out_buffer(out, sl.mr_out, bytes);
    launch_residual(Launch{sl.stream, &sl.launches}, c, d, M, N, origin(it, nsub, nmesh, nshell),
                    origin(jt, nsub, nmesh, nshell), origin(kt, nsub, nmesh, nshell), next, seed);
    finish_out(out, d, bytes, sl.stream);
    PPB_CUDA(cudaStreamSynchronize(sl.stream));
  });
}

int32_t ppb_interpolate_to_tile(ppb_ctx* ctx, const float* coarse, int32_t it, int32_t jt, int32_t kt, int32_t nsub,
                                int32_t nmesh, int64_t N, int32_t M, float* out) {
  return guarded(ctx, [&] {
    PPB_REQUIRE(coarse && out, "null argument");
    check_coarse(N, M);
    check_tile(it, jt, kt, nsub, nmesh);
    Slot& sl = ctx->sync;
    const size_t bytes = (size_t)nmesh * nmesh * nmesh * 4;
    const float* c = (const float*)stage_in(sl.mr_in, coarse, (size_t)M * M * M * 4, sl.stream);
    float* d = out_buffer(out, sl.mr_out, bytes);
    Launch L{sl.stream, &sl.launches};
    sl.mr_axis.ensure((size_t)3 * nmesh * 32);
    int4* aidx = sl.mr_axis.as<int4>();
    float4* awt = reinterpret_cast<float4*>(aidx + 3 * nmesh);
    launch_axis_weights(L, aidx, awt, M, N, origin(it, nsub, nmesh, 0), origin(jt, nsub, nmesh, 0),
                        origin(kt, nsub, nmesh, 0), nmesh);
    launch_tricubic(L, aidx, awt, M, nmesh, 1, c, &d, nullptr, 0, 0, 0);
    finish_out(out, d, bytes, sl.stream);
    PPB_CUDA(cudaStreamSynchronize(sl.stream));
  });
}

int32_t ppb_isolated_convolve(ppb_ctx* ctx, const float* noise, int32_t n_input, double boxsize_local, int32_t n,
                              const int32_t* kernels, int32_t nkern, int32_t nshell, float* out) {
  return guarded(ctx, [&] {
    PPB_REQUIRE(noise && out && kernels, "null argument");
    PPB_REQUIRE(n_input >= 1 && n_input <= 640, "n_input must be 1..640");
    PPB_REQUIRE(n >= 1 && nshell >= 0 && (int64_t)nshell + n <= 2 * (int64_t)n_input,
                "the tile region [nshell, nshell + n) must lie inside the padded box");
    PPB_REQUIRE(nkern >= 1 && nkern <= 64, "nkern must be 1..64");
    PPB_REQUIRE(boxsize_local > 0.0, "boxsize_local must be > 0");
    for (int b = 0; b < nkern; b++) check_kernel(kernels[3 * b], kernels[3 * b + 1], kernels[3 * b + 2]);
    std::shared_lock<std::shared_mutex> rl(ctx->sh.mu);
    PPB_REQUIRE(ctx->sh.pk_n >= 2, "P(k) table not set (ppb_set_pk_table)");
    Slot& sl = ctx->sync;
    cudaStream_t s = sl.stream;
    const int64_t Nt = (int64_t)n * n * n;
    const float* src = (const float*)stage_in(sl.mr_in, noise, (size_t)n_input * n_input * n_input * 4, s);
    float* dout = out_buffer(out, sl.mr_out, (size_t)nkern * Nt * 4);
    std::vector<float*> outs(nkern);
    for (int b = 0; b < nkern; b++) outs[b] = dout + b * Nt;
    mr_isolated_device(ctx, sl, src, n_input, boxsize_local, n, kernels, nkern, nshell, outs.data());
    finish_out(out, dout, (size_t)nkern * Nt * 4, s);
    PPB_CUDA(cudaStreamSynchronize(s));
  });
}

int32_t ppb_compute_2lpt(ppb_ctx* ctx, const float* delta_tile, int32_t n, double boxsize_local, float* psi2) {
  return guarded(ctx, [&] {
    PPB_REQUIRE(delta_tile && psi2, "null argument");
    PPB_REQUIRE(n >= 2 && n <= 1024, "n must be 2..1024");
    PPB_REQUIRE(boxsize_local > 0.0, "boxsize_local must be > 0");
    Slot& sl = ctx->sync;
    const int64_t N = (int64_t)n * n * n;
    TileRes& tr = periodic_setup(ctx, delta_tile, n);
    float* d = out_buffer(psi2, sl.mr_out, (size_t)3 * N * 4);
    mr_tile_2lpt_lap(ctx, sl, tr, n, boxsize_local, d, nullptr);
    finish_out(psi2, d, (size_t)3 * N * 4, sl.stream);
    PPB_CUDA(cudaStreamSynchronize(sl.stream));
  });
}

int32_t ppb_compute_laplacian(ppb_ctx* ctx, const float* delta_tile, int32_t n, double boxsize_local, float* lapd) {
  return guarded(ctx, [&] {
    PPB_REQUIRE(delta_tile && lapd, "null argument");
    PPB_REQUIRE(n >= 2 && n <= 1024, "n must be 2..1024");
    PPB_REQUIRE(boxsize_local > 0.0, "boxsize_local must be > 0");
    Slot& sl = ctx->sync;
    const int64_t N = (int64_t)n * n * n;
    TileRes& tr = periodic_setup(ctx, delta_tile, n);
    float* d = out_buffer(lapd, sl.mr_out, (size_t)N * 4);
    mr_tile_2lpt_lap(ctx, sl, tr, n, boxsize_local, nullptr, d);
    finish_out(lapd, d, (size_t)N * 4, sl.stream);
    PPB_CUDA(cudaStreamSynchronize(sl.stream));
  });
}

int32_t ppb_coarse_fields(ppb_ctx* ctx, const float* coarse_noise, int32_t M, double boxsize_full, int32_t ilpt,
                          int32_t ioutshear, float* delta, float* psi, float* psi2, float* lapd) {
  return guarded(ctx, [&] {
    PPB_REQUIRE(coarse_noise, "null argument");
    PPB_REQUIRE(M >= 2 && M <= 1024, "M must be 2..1024");
    PPB_REQUIRE(boxsize_full > 0.0, "boxsize_full must be > 0");
    std::shared_lock<std::shared_mutex> rl(ctx->sh.mu);
    PPB_REQUIRE(ctx->sh.pk_n >= 2, "P(k) table not set (ppb_set_pk_table)");
    Slot& sl = ctx->sync;
    cudaStream_t s = sl.stream;
    const int64_t N = (int64_t)M * M * M;
    const float* src = (const float*)stage_in(sl.mr_in, coarse_noise, (size_t)N * 4, s);
    // outputs: delta, psi (3), psi2 (3), lapd, each starting on a 16-byte
    // boundary (cuFFT's real output must be aligned to its complex type)
    const int64_t fs = (N + 3) & ~(int64_t)3;
    sl.mr_aux.ensure(8 * fs * 4);
    float* o = sl.mr_aux.as<float>();
    mr_coarse_device(ctx, sl, src, M, boxsize_full, ilpt, ioutshear, o, fs);
    if (delta) copy_out(delta, o, N * 4, s);
    for (int q = 0; q < 3; q++) {
      if (psi) copy_out(psi + q * N, o + (1 + q) * fs, N * 4, s);
      if (psi2 && ilpt >= 2) copy_out(psi2 + q * N, o + (4 + q) * fs, N * 4, s);
    }
    if (lapd && ioutshear >= 1) copy_out(lapd, o + 7 * fs, N * 4, s);
    PPB_CUDA(cudaStreamSynchronize(s));
  });
}

}  // extern "C"
