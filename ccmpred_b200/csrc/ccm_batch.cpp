// Many alignments solved to convergence concurrently: a pool of host worker
// threads, each driving its own context (and CUDA stream) through the
// reweighting, init_bias, the device conjugate gradient and the APC contact
// map.  Alignments are handed out largest-first (cost ~ N L^2) so that the
// long solves start early.  Small alignments leave most of the GPU idle on
// their own; running several at once on separate streams fills it.  The
// parameter vector x of each solve lives on the device only (the host sends
// the 20 L single fields and receives the L x L contact map), device memory is
// allocated and freed stream-ordered from one pool that keeps it mapped, and
// pinned records come from a never-freed slab: no worker's set-up or tear-down
// waits for the whole device or moves the full x over PCIe.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "ccm_internal.cuh"
#include "ccm_layout.cuh"

size_t ccm::context_bytes_estimate(int L, int N, int path) {
  const size_t Np = ((size_t)N + 255) / 256 * 256, QL = (size_t)kQ * L;
  size_t b = (size_t)N * L + 4 * (size_t)N + 4096;  // alignment, weights, result
  if (path == CCM_PATH_TC_I8SP) {
    const size_t T = ((size_t)L + 8) / 9, SW = 192 * T, S = (SW + 255) / 256 * 256;
    const size_t KP = (QL + 255) / 256 * 256;
    b += 5 * Np * S + 3 * KP * SW + Np * KP + Np * KP / 8 + 8 * (Np / 128) * T * 8;
    b += 4 * (QL + S);
  } else if (path == CCM_PATH_TC_I8X3) {
    const size_t S = 256 * (((size_t)L + kGroupCols - 1) / kGroupCols);
    b += 5 * Np * S + 3 * S * S + 8 * (Np / 128) * (S / 256) * 8 + 4 * (QL + S);
  } else if (path == CCM_PATH_TC_BF16X2 || path == CCM_PATH_TC_BF16X3) {
    const size_t ns = path == CCM_PATH_TC_BF16X3 ? 3 : 2;
    const size_t S = 256 * (((size_t)L + kGroupCols - 1) / kGroupCols);
    b += 2 * Np * S + ns * 2 * (S * S + Np * S) + 8 * (Np / 128) * (S / 256) * 8;
  } else {
    const size_t elem = path == CCM_PATH_SIMT_F64 ? 8 : 4;
    b += elem * ((size_t)N * QL + QL * QL + QL) + 8 * ((size_t)N + QL);
  }
  const size_t blocks = (QL + 255) / 256 + 1;
  b += 8 * QL + 4 * QL + 8 * blocks * blocks;  // partials, g1, backward tile list
  return b + (8u << 20);                      // pool granularity
}

namespace {

// One alignment of a wave.
struct WaveItem {
  int i = 0;
  ccm_context *ctx = nullptr;
  float *d_x = nullptr, *d_map = nullptr;
  ccm::CgGraphSolve *gs = nullptr;
};

// Alignments in waves, each wave ONE graph launch: the contexts and device x of a
// wave are set up on one stream, then every alignment's whole device-side solve
// (initial evaluation, the iteration loop in conditional nodes, the final x) and
// its contact-score kernel go into one graph as independent branches; the graph
// runs them concurrently and the host waits once per wave.  Waves are filled
// largest-first up to a device-memory budget and a count.
int solve_waves(int n, const ccm_msa_desc *msas, const ccm_batch_params *params,
                ccm_batch_result *results, float **contact_maps, const std::vector<int> &order) {
  using namespace ccm;
  (void)n;
  const int dev = params->device;
  if (cudaSetDevice(dev) != cudaSuccess)
    return set_last_error(CCM_ERR_CUDA, "ccm_solve_batch: cannot select device %d", dev);
  size_t mem_free = 0, mem_total = 0;
  cudaMemGetInfo(&mem_free, &mem_total);
  const size_t budget = params->wave_bytes > 0 ? params->wave_bytes : mem_free / 10 * 6;
  const int wave_max = params->wave_max > 0 ? params->wave_max : 64;
  cudaMemPool_t pool = nullptr;
  {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess)
      return set_last_error(CCM_ERR_CUDA, "ccm_solve_batch: cannot create a memory pool");
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaStream_t stream = nullptr;
  if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaMemPoolDestroy(pool);
    return set_last_error(CCM_ERR_CUDA, "ccm_solve_batch: cannot create a stream");
  }
  int rc = CCM_OK;
  size_t pos = 0;
  while (rc == CCM_OK && pos < order.size()) {
    // the wave: largest-first, within the memory budget (at least one alignment)
    std::vector<WaveItem> wave;
    size_t bytes = 0;
    while (pos < order.size() && (int)wave.size() < wave_max) {
      const ccm_msa_desc &m = msas[order[pos]];
      const size_t need = context_bytes_estimate(m.ncol, m.nrow, m.path >= 0 ? m.path : params->path) +
                          5 * sizeof(float) * (size_t)ccm_nvar_padded(m.ncol) +
                          sizeof(float) * (size_t)m.ncol * m.ncol;
      if (!wave.empty() && bytes + need > budget) break;
      bytes += need;
      WaveItem it;
      it.i = order[pos++];
      wave.push_back(it);
    }
    const auto t0 = std::chrono::steady_clock::now();
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaError_t e = cudaGraphCreate(&graph, 0);
    if (e != cudaSuccess) rc = set_last_error(CCM_ERR_CUDA, "ccm_solve_batch: %s", cudaGetErrorString(e));
    for (WaveItem &it : wave) {
      if (rc != CCM_OK) break;
      const ccm_msa_desc &m = msas[it.i];
      const int L = m.ncol, N = m.nrow;
      std::vector<float> w(N, 1.0f);
      if (params->reweighting_threshold < 1.0f)
        rc = ccm_calculate_weights(m.msa, L, N, params->reweighting_threshold, w.data(), dev);
      const long long nv = ccm_nvar_padded(L), nsp = ccm_nsingle_padded(L);
      std::vector<float> x1((size_t)nsp, 0.0f);
      if (rc == CCM_OK) {
        // x lives on the device only: the host computes the single fields of
        // init_bias (20 L floats) and the couplings start at zero
        init_single_fields(m.msa, L, N, x1.data());
        ccm_options o;
        ccm_options_default(&o, L);
        o.lambda_single = params->lambda_single;
        o.lambda_pair = params->lambda_pair_factor * (float)(L - 1);
        o.path = m.path >= 0 ? m.path : params->path;
        o.device = dev;
        o.stream = stream;
        rc = create_context(&it.ctx, m.msa, L, N, w.data(), &o, pool);
      }
      if (rc == CCM_OK) {
        e = dev_alloc_raw(it.ctx, reinterpret_cast<void **>(&it.d_x), sizeof(float) * (size_t)nv);
        if (e == cudaSuccess)
          e = cudaMemsetAsync(it.d_x + nsp, 0, sizeof(float) * (size_t)(nv - nsp), stream);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(it.d_x, x1.data(), sizeof(float) * (size_t)nsp, cudaMemcpyHostToDevice,
                              stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);  // x1 is a host temporary
        if (e == cudaSuccess && contact_maps && contact_maps[it.i])
          e = dev_alloc_raw(it.ctx, reinterpret_cast<void **>(&it.d_map),
                            sizeof(float) * (size_t)L * L);
        if (e != cudaSuccess)
          rc = set_last_error(e == cudaErrorMemoryAllocation ? CCM_ERR_NOMEM : CCM_ERR_CUDA,
                              "ccm_solve_batch: %s", cudaGetErrorString(e));
      }
      cudaGraphNode_t last = nullptr;
      if (rc == CCM_OK) rc = cg_graph_solve_add(it.ctx, it.d_x, &params->cg, graph, &it.gs, &last);
      if (rc == CCM_OK && it.d_map) {
        // the contact scores after the solve, in the same branch
        e = cudaStreamBeginCaptureToGraph(stream, graph, &last, nullptr, 1,
                                          cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
          e = launch_contact_scores(it.d_x, it.d_map, L, stream);
          cudaGraph_t tmp = nullptr;
          const cudaError_t e2 = cudaStreamEndCapture(stream, &tmp);
          if (e == cudaSuccess) e = e2;
        }
        if (e != cudaSuccess) rc = set_last_error(CCM_ERR_CUDA, "ccm_solve_batch: %s", cudaGetErrorString(e));
      }
    }
    if (rc == CCM_OK) {
      e = cudaStreamSynchronize(stream);  // contexts and x set up before the launch
      if (e == cudaSuccess && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
        rc = set_last_error(CCM_ERR_UNSUPPORTED, "ccm_solve_batch: the wave's graph");
      if (e == cudaSuccess && rc == CCM_OK) e = cudaGraphLaunch(exec, stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
      if (e != cudaSuccess) rc = set_last_error(CCM_ERR_CUDA, "ccm_solve_batch: %s", cudaGetErrorString(e));
    }
    const double secs =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (WaveItem &it : wave) {
      ccm_batch_result &r = results[it.i];
      std::memset(&r, 0, sizeof(r));
      r.seconds = secs;  // the wave's wall time: its alignments run together
      if (rc == CCM_OK && it.gs) {
        ccm_cg_result cg;
        const int rr = cg_graph_solve_result(it.gs, &cg);
        r.status = rr == CCM_OK ? cg.status : rr;
        r.iterations = cg.iterations;
        r.evaluations = cg.evaluations;
        r.fx = cg.fx;
        if (rr != CCM_OK) rc = rr;
        if (rr == CCM_OK && it.d_map) {
          const int L = msas[it.i].ncol;
          e = cudaMemcpy(contact_maps[it.i], it.d_map, sizeof(float) * (size_t)L * L,
                         cudaMemcpyDeviceToHost);
          if (e != cudaSuccess) rc = set_last_error(CCM_ERR_CUDA, "ccm_solve_batch: %s", cudaGetErrorString(e));
          else if (params->use_apc) ccm_apc(contact_maps[it.i], L);
        }
      } else {
        r.status = rc != CCM_OK ? rc : CCM_ERR_CUDA;
      }
      cg_graph_solve_free(it.gs);
      if (it.d_map) cudaFreeAsync(it.d_map, stream);
      if (it.d_x) cudaFreeAsync(it.d_x, stream);
      if (it.ctx) ccm_destroy(it.ctx);
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
  cudaStreamSynchronize(stream);
  cudaStreamDestroy(stream);
  cudaMemPoolDestroy(pool);
  return rc;
}

}  // namespace

extern "C" {

void ccm_batch_params_default(ccm_batch_params *p) {
  if (!p) return;
  p->reweighting_threshold = 0.8f;
  p->lambda_single = 0.01f;
  p->lambda_pair_factor = 0.2f;
  p->path = CCM_PATH_TC_I8SP;
  p->workers = 8;
  p->device = 0;
  p->use_apc = 1;
  p->sms_per_worker = 0;
  p->waves = 0;
  p->wave_max = 64;
  p->wave_bytes = 0;
  ccm_cg_params_default(&p->cg);
}

int ccm_solve_batch(int n, const ccm_msa_desc *msas, const ccm_batch_params *params,
                    ccm_batch_result *results, float **contact_maps) {
  if (n < 0 || (n > 0 && (!msas || !results)) || !params || params->workers < 1) return CCM_ERR_INVALID;
  for (int i = 0; i < n; ++i)
    if (!msas[i].msa || msas[i].ncol <= 0 || msas[i].nrow <= 0 || msas[i].path > CCM_PATH_TC_I8SP ||
        msas[i].path == CCM_PATH_SIMT_F64)
      return CCM_ERR_INVALID;
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::sort(order.begin(), order.end(), [&](int a, int b) {
    const double ca = (double)msas[a].nrow * msas[a].ncol * msas[a].ncol;
    const double cb = (double)msas[b].nrow * msas[b].ncol * msas[b].ncol;
    return ca > cb;
  });
  if (params->waves) {
    const int rc = solve_waves(n, msas, params, results, contact_maps, order);
    if (rc != CCM_ERR_UNSUPPORTED) return rc;
    // nested conditional nodes refused by this driver: host worker threads
    (void)cudaGetLastError();
  }
  const int nw = std::min(params->workers, std::max(n, 1));
  // An optional share of the SMs for each worker's contexts.  Measured on B200,
  // no share is faster: the prep and CG kernels spread over every SM anyway,
  // so a share only shrinks the GEMM grids.
  const int max_sms = params->sms_per_worker > 0 ? params->sms_per_worker : 0;
  // One memory pool for the whole batch that keeps freed blocks mapped: each
  // alignment's buffers reuse the previous alignment's memory instead of
  // mapping fresh device memory (the default pool gives it back at every
  // synchronisation).  Destroyed when the batch ends.
  cudaMemPool_t pool = nullptr;
  {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = params->device;
    if (cudaSetDevice(params->device) != cudaSuccess || cudaMemPoolCreate(&pool, &props) != cudaSuccess)
      return ccm::set_last_error(CCM_ERR_CUDA, "ccm_solve_batch: cannot create a memory pool");
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  std::atomic<int> next(0);
  std::atomic<int> first_error(CCM_OK);
  std::mutex err_mutex;
  std::string err_text;

  auto work = [&]() {
    cudaSetDevice(params->device);
    // a non-blocking stream per worker: no implicit ordering with the legacy
    // default stream, which would interfere with the CG's graph capture while
    // other workers are running
    cudaStream_t stream = nullptr;
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
      int expected = CCM_OK;
      first_error.compare_exchange_strong(expected, CCM_ERR_CUDA);
      std::lock_guard<std::mutex> lock(err_mutex);
      err_text = "ccm_solve_batch: cannot create a worker stream";
      return;
    }
    for (;;) {
      const int slot = next.fetch_add(1);
      if (slot >= n || first_error.load() != CCM_OK) break;
      const int i = order[slot];
      const ccm_msa_desc &m = msas[i];
      ccm_batch_result &r = results[i];
      std::memset(&r, 0, sizeof(r));
      const auto t0 = std::chrono::steady_clock::now();
      const int L = m.ncol, N = m.nrow;
      std::vector<float> w(N, 1.0f);
      int rc = CCM_OK;
      if (params->reweighting_threshold < 1.0f)
        rc = ccm_calculate_weights(m.msa, L, N, params->reweighting_threshold, w.data(),
                                   params->device);
      // x lives on the device only: the host computes the single fields of
      // init_bias (20 L floats) and the couplings start at zero
      const long long nv = ccm_nvar_padded(L), nsp = ccm_nsingle_padded(L);
      std::vector<float> x1(rc == CCM_OK ? (size_t)nsp : 0, 0.0f);
      ccm_context *ctx = nullptr;
      float *d_x = nullptr, *d_map = nullptr;
      if (rc == CCM_OK) {
        ccm::init_single_fields(m.msa, L, N, x1.data());
        ccm_options o;
        ccm_options_default(&o, L);
        o.lambda_single = params->lambda_single;
        o.lambda_pair = params->lambda_pair_factor * (float)(L - 1);
        o.path = m.path >= 0 ? m.path : params->path;
        o.device = params->device;
        o.stream = stream;
        o.max_sms = max_sms;
        rc = ccm::create_context(&ctx, m.msa, L, N, w.data(), &o, pool);
      }
      auto cuda_ok = [&](cudaError_t e) {
        if (e != cudaSuccess && rc == CCM_OK)
          rc = ccm::set_last_error(CCM_ERR_CUDA, "ccm_solve_batch: %s", cudaGetErrorString(e));
        return rc == CCM_OK;
      };
      if (rc == CCM_OK && cuda_ok(ccm::dev_alloc_raw(ctx, reinterpret_cast<void **>(&d_x),
                                                      sizeof(float) * (size_t)nv)) &&
          cuda_ok(cudaMemsetAsync(d_x + nsp, 0, sizeof(float) * (size_t)(nv - nsp), stream)))
        cuda_ok(cudaMemcpyAsync(d_x, x1.data(), sizeof(float) * (size_t)nsp,
                                cudaMemcpyHostToDevice, stream));
      ccm_cg_result cg;
      std::memset(&cg, 0, sizeof(cg));
      if (rc == CCM_OK) rc = ccm_conjugrad_gpu(ctx, d_x, nv, &params->cg, nullptr, nullptr, &cg);
      if (rc == CCM_OK && contact_maps && contact_maps[i]) {
        // contact scores on the device (bit-identical to the host sum_submatrices);
        // only the L x L map comes back
        const size_t mb = sizeof(float) * (size_t)L * L;
        if (cuda_ok(ccm::dev_alloc_raw(ctx, reinterpret_cast<void **>(&d_map), mb)) &&
            cuda_ok(ccm::launch_contact_scores(d_x, d_map, L, stream)) &&
            cuda_ok(cudaMemcpyAsync(contact_maps[i], d_map, mb, cudaMemcpyDeviceToHost, stream)) &&
            cuda_ok(cudaStreamSynchronize(stream)) && params->use_apc)
          ccm_apc(contact_maps[i], L);
      }
      if (d_map) cudaFreeAsync(d_map, stream);
      if (d_x) cudaFreeAsync(d_x, stream);
      if (ctx) ccm_destroy(ctx);
      r.status = rc == CCM_OK ? cg.status : rc;
      r.iterations = cg.iterations;
      r.evaluations = cg.evaluations;
      r.fx = cg.fx;
      r.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      if (rc != CCM_OK) {
        int expected = CCM_OK;
        if (first_error.compare_exchange_strong(expected, rc)) {
          std::lock_guard<std::mutex> lock(err_mutex);
          err_text = std::string("alignment ") + std::to_string(i) + ": " + ccm_last_error();
        }
      }
    }
    cudaStreamDestroy(stream);
  };
  std::vector<std::thread> threads;
  for (int t = 0; t < nw; ++t) threads.emplace_back(work);
  for (auto &t : threads) t.join();
  // every allocation has been freed on its worker's stream; the pool's memory
  // is released once those frees have completed
  cudaMemPoolDestroy(pool);
  const int rc = first_error.load();
  if (rc != CCM_OK) ccm::set_last_error(rc, "ccm_solve_batch: %s", err_text.c_str());
  return rc;
}

}  // extern "C"
