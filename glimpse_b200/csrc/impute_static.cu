// gp_impute_one_static: the imputation forward-backward for one haplotype with
// every piece of device scratch carved out of one fixed region that is part of
// the library image, so that the call itself allocates no device memory.
//
// Some callers cannot allocate device memory when they want a posterior:
//   * a host process whose device memory is already handed out (another
//     framework's caching allocator, or a service held to a fixed footprint
//     after start-up) would see cudaMalloc fail or push that owner into a
//     release;
//   * a caller that imputes one haplotype at a time on a latency-bound path
//     would pay for cudaMalloc, and cudaFree waits for the whole device,
//     serialising it against every other stream in the process.
// For them this entry point takes its scratch from g_impute_scratch below. The
// region is fixed at kStaticScratchBytes per device. The per-site buffers are
// sized on all L sites, and a call whose per-site buffers do not fit is refused
// with GP_E_ARG before any work is queued. The forward-backward store takes the
// rest of the region; it needs (polymorphic sites of the conditioning set) x
// (row stride) x 4 bytes, which is known only once the conditioning set is
// built on the device, so a call whose store does not fit is refused with
// GP_E_ARG after that step and before the HMM runs.
//
// The region's address is looked up once per device, the first time the entry
// is called with that device current (cudaGetSymbolAddress); that first call
// therefore does set-up work, and it should be made before any stream capture
// begins. There is one region per device and no lock: calls that overlap on
// the same device (two host threads, or two contexts on one device whose
// streams run concurrently) use the same bytes and race.
//
// The kernels are the ones gp_impute_batch launches, in the same order; only
// where their buffers live differs.
#include <cuda_runtime.h>

#include <atomic>

#include "context.h"
#include "internal.h"

namespace gp {
namespace {

constexpr size_t kStaticScratchBytes = size_t(64) << 20;  // 64 MiB per device
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_impute_scratch[kStaticScratchBytes];

std::atomic<unsigned char*> g_scratch_addr[kMaxDevices] = {};

size_t round256(size_t x) { return (x + 255) & ~size_t(255); }

// Byte offsets of every buffer of a one-haplotype imputation inside the region.
// The per-site buffers are sized on all L sites; the forward-backward store
// starts at `alpha` and may use the region up to its end.
struct StaticLayout {
  size_t states, nstates, mark, polyidx, poly, npoly, hvar, em, tr, fl, alpha_off, split, split_scr, hl, hp, flat,
      alpha;
};

StaticLayout static_layout(int L, int Kp, int Ks) {
  const int WB = (L + 31) / 32;
  StaticLayout s{};
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t at = o;
    o += round256(bytes);
    return at;
  };
  s.states = take((size_t)Kp * 4);
  s.nstates = take(4);
  s.mark = take((size_t)L);
  s.polyidx = take((size_t)L * 4);
  s.poly = take((size_t)L * 4);
  s.npoly = take(4);
  s.hvar = take((size_t)WB * Kp * 4);
  s.em = take((size_t)L * 16);
  s.tr = take((size_t)L * 8);
  s.fl = take((size_t)L);
  s.alpha_off = take(8);
  s.split = take(4);
  s.split_scr = take((size_t)(4 + Ks) * 4);
  s.hl = take((size_t)L * 2 * 4);
  s.hp = take((size_t)L * 2 * 4);
  s.flat = take((size_t)L);
  s.alpha = o;
  return s;
}

void point(DevBuf& b, unsigned char* base, size_t off, size_t bytes) {
  b.ptr = base + off;
  b.cap = bytes;
}

}  // namespace
}  // namespace gp

using gp::Context;

extern "C" int gp_impute_one_static(gp_ctx* ctx, int32_t k, const uint32_t* states, const float* hl,
                                    const uint8_t* flat, float* hp) {
  if (!ctx) return GP_E_ARG;
  Context& c = *reinterpret_cast<Context*>(ctx);
  if (k <= 0 || !states || !hl || !flat || !hp) return (c.fail(GP_E_ARG, "impute_one_static: bad argument"), GP_E_ARG);
  if (k > gp::kMaxStates)
    return (c.fail(GP_E_ARG, "impute_one_static: more than 2048 states"), GP_E_ARG);
  for (int j = 0; j < k; ++j) {
    if ((int)states[j] >= c.panel.N) return (c.fail(GP_E_ARG, "impute_one_static: state id out of range"), GP_E_ARG);
    if (j > 0 && states[j - 1] >= states[j])
      return (c.fail(GP_E_ARG, "impute_one_static: state ids must be sorted and unique"), GP_E_ARG);
  }
  const int L = c.panel.L;
  const int Kp = (k + 31) / 32 * 32;
  const int Ks = gp::impute_store_stride(k);
  const gp::StaticLayout lay = gp::static_layout(L, Kp, Ks);
  if (lay.alpha + (size_t)Ks * 4 * 32 > gp::kStaticScratchBytes)
    return (c.fail(GP_E_ARG, "impute_one_static: the per-site buffers of " + std::to_string(L) + " sites x " +
                                 std::to_string(k) + " states need " + std::to_string(lay.alpha >> 20) +
                                 " MiB of scratch, above the fixed 64 MiB"),
            GP_E_ARG);
  const size_t store_cap = gp::kStaticScratchBytes - lay.alpha;
  const int dev = c.cfg.device;
  if (dev < 0 || dev >= gp::kMaxDevices) return (c.fail(GP_E_ARG, "impute_one_static: device ordinal"), GP_E_ARG);

  int prev = -1;
  cudaError_t e = cudaGetDevice(&prev);
  if (e != cudaSuccess) return c.cuda_fail(e, "impute_one_static: current device");
  if (prev != dev && (e = cudaSetDevice(dev)) != cudaSuccess) return c.cuda_fail(e, "impute_one_static: set device");
  auto finish = [&](int rc) {
    if (prev != dev) cudaSetDevice(prev);
    return rc;
  };
  // Per-device set-up: the region's device address, looked up with the device current.
  unsigned char* base = gp::g_scratch_addr[dev].load(std::memory_order_acquire);
  if (!base) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, gp::g_impute_scratch);
    if (e != cudaSuccess || !p) return finish(c.cuda_fail(e, "impute_one_static: scratch symbol address"));
    base = static_cast<unsigned char*>(p);
    gp::g_scratch_addr[dev].store(base, std::memory_order_release);
  }

  gp::ImputeWork w;
  w.n = 1;
  w.L = L;
  w.Kp = Kp;
  w.WB = (L + 31) / 32;
  w.Ks = Ks;
  gp::point(w.states, base, lay.states, (size_t)Kp * 4);
  gp::point(w.nstates, base, lay.nstates, 4);
  gp::point(w.mark, base, lay.mark, L);
  gp::point(w.polyidx, base, lay.polyidx, (size_t)L * 4);
  gp::point(w.poly, base, lay.poly, (size_t)L * 4);
  gp::point(w.npoly, base, lay.npoly, 4);
  gp::point(w.hvar, base, lay.hvar, (size_t)w.WB * Kp * 4);
  gp::point(w.em, base, lay.em, (size_t)L * 16);
  gp::point(w.tr, base, lay.tr, (size_t)L * 8);
  gp::point(w.fl, base, lay.fl, L);
  gp::point(w.alpha_off, base, lay.alpha_off, 8);
  gp::point(w.split, base, lay.split, 4);
  gp::point(w.split_scr, base, lay.split_scr, (size_t)(4 + Ks) * 4);
  gp::point(w.alpha, base, lay.alpha, store_cap);
  gp::point(w.hl, base, lay.hl, (size_t)L * 8);
  gp::point(w.hp, base, lay.hp, (size_t)L * 8);
  gp::point(w.flat, base, lay.flat, L);

  cudaStream_t s = c.stream;
  const int32_t kk = k;
  const int64_t zero64 = 0;
  // The state list is padded to Kp entries; the padding starts at zero.
  cudaMemsetAsync(w.states.ptr, 0, (size_t)Kp * 4, s);
  cudaMemcpyAsync(w.states.ptr, states, (size_t)k * 4, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(w.nstates.ptr, &kk, 4, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(w.hl.ptr, hl, (size_t)L * 8, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(w.flat.ptr, flat, (size_t)L, cudaMemcpyHostToDevice, s);
  gp::launch_mark_poly(c.panel, w, s);
  gp::launch_compact_poly(c.panel, w, s);
  gp::launch_build_hvar(c.panel, w, s);
  int32_t np = 0;
  cudaMemcpyAsync(&np, w.npoly.ptr, 4, cudaMemcpyDeviceToHost, s);
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return finish(c.cuda_fail(e, "impute_one_static: conditioning set"));
  if ((size_t)np * Ks * 4 > store_cap)
    return finish((c.fail(GP_E_ARG, "impute_one_static: " + std::to_string(np) + " polymorphic sites x " +
                                        std::to_string(k) + " states need a " +
                                        std::to_string(((size_t)np * Ks * 4) >> 20) +
                                        " MiB forward-backward store; the fixed 64 MiB region has " +
                                        std::to_string(store_cap >> 20) + " MiB left for it"),
                   GP_E_ARG));
  const int32_t split = (np / 2) & ~31;  // forward/backward meeting point, a multiple of 32
  cudaMemcpyAsync(w.alpha_off.ptr, &zero64, 8, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(w.split.ptr, &split, 4, cudaMemcpyHostToDevice, s);
  gp::launch_site_records(c.panel, c.mc, w, w.hl.as<float>(), w.flat.as<uint8_t>(), s);
  const int J = gp::impute_groups(k);
  int lrc = gp::launch_impute_warp(1, J, c.mc, w, w.hp.as<float>(), s);
  if (lrc == GP_OK) lrc = gp::launch_impute_warp(2, J, c.mc, w, w.hp.as<float>(), s);
  if (lrc == GP_E_CUDA) return finish(c.cuda_fail(cudaGetLastError(), "impute_one_static: shared-memory attribute"));
  if (lrc != GP_OK) return finish((c.fail(GP_E_ARG, "impute_one_static: too many states"), GP_E_ARG));
  gp::launch_impute_finish(c.panel, c.mc, w, w.hl.as<float>(), w.flat.as<uint8_t>(), w.hp.as<float>(), s);
  c.prof.kernel_launches += 9;
  cudaMemcpyAsync(hp, w.hp.ptr, (size_t)L * 8, cudaMemcpyDeviceToHost, s);
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return finish(c.cuda_fail(e, "impute_one_static"));
  if ((e = cudaGetLastError()) != cudaSuccess) return finish(c.cuda_fail(e, "impute_one_static: launch"));
  return finish(GP_OK);
}
