// extern "C" entry points declared in include/mc3.h.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include <string>

#include "dft_gemm.cuh"
#include "engine.h"
#include "profile.h"
#include "proposal.h"
#include "queue.h"

struct mc3_proposal {
  int gpu;
  mc3::proposal::Net net;
};

struct mc3_ctx {
  mc3::Engine* eng;
  mc3::MovieQueue* queue = nullptr;  // created by the first mc3_submit
};

using namespace mc3;

namespace {
cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }
}  // namespace

extern "C" {

const char* mc3_version(void) { return "mc3-b200 0.1.0 (MotionCor3 1.2.1 hot path, sm_100a)"; }

const char* mc3_strerror(int code) {
  switch (code) {
    case MC3_OK: return "ok";
    case MC3_EINVAL: return "invalid argument or size";
    case MC3_ENOMEM: return "out of memory";
    case MC3_ECUDA: return "CUDA runtime error";
    case MC3_ETIMEOUT: return "device wait timed out";
    case MC3_EIO: return "file I/O error";
    case MC3_EUNSUPPORTED: return "unsupported option or size";
    case MC3_ETOOBIG: return "size exceeds the fixed scratch of the no-allocation entry point";
    default: return "unknown error";
  }
}

void mc3_params_default(mc3_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  // CInput::CInput (CInput.cpp:82-127)
  p->patch[0] = p->patch[1] = p->patch[2] = 0;
  p->iter = 15;
  p->tol = 0.1f;
  p->bft[0] = 500.0f;
  p->bft[1] = 100.0f;
  p->phase_only = 0;
  p->ft_bin = 1.0f;
  p->init_dose = 0.0f;
  p->fm_dose = 0.0f;
  p->pix_size = 0.0f;
  p->kv = 300;
  p->group[0] = 1;
  p->group[1] = 4;
  p->fm_ref = -1;
  p->sum_range[0] = 3.0f;
  p->sum_range[1] = 25.0f;
  p->align = 1;
  p->correct_bad = 1;
  p->gpu = 0;
  p->split_sum = 0;
  p->out_stack[0] = 0;
  p->out_stack[1] = 1;
  p->mag[0] = 1.0f;
  p->mag[1] = 1.0f;
  p->mag[2] = 0.0f;
  p->in_fm_motion = 0;
  p->corr_interp = 0;
  p->cs = 0.0f;
  p->amp_cont = 0.07f;
  p->ext_phase = 0.0f;
  p->dft_gemm = 0;
}

int mc3_create(const mc3_params* p, mc3_ctx** out) {
  if (!p || !out) return MC3_EINVAL;
  *out = nullptr;
  if (p->iter < 1 || p->group[0] < 1 || p->group[1] < 1) return MC3_EINVAL;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return MC3_ECUDA;
  }
  if (p->gpu < 0 || p->gpu >= ndev) return MC3_EINVAL;
  mc3_ctx* c = new (std::nothrow) mc3_ctx;
  if (!c) return MC3_ENOMEM;
  c->eng = new (std::nothrow) Engine(*p);
  if (!c->eng) {
    delete c;
    return MC3_ENOMEM;
  }
  int s = c->eng->init();
  if (s != kOk) {
    delete c->eng;
    delete c;
    return s;
  }
  *out = c;
  return MC3_OK;
}

int mc3_destroy(mc3_ctx* ctx) {
  if (!ctx) return MC3_EINVAL;
  delete ctx->queue;  // finishes the queued movies first
  delete ctx->eng;
  delete ctx;
  return MC3_OK;
}

int mc3_set_stream(mc3_ctx* ctx, void* stream) {
  if (!ctx) return MC3_EINVAL;
  return ctx->eng->set_stream(as_stream(stream));
}

namespace {
bool queue_busy(mc3_ctx* ctx);
}  // namespace

int mc3_plan(mc3_ctx* ctx, int nx, int ny, int nz, mc3_plan_info* info) {
  if (!ctx || !info) return MC3_EINVAL;
  // while movies are queued the worker owns the buffers: sizes only
  if (queue_busy(ctx)) return ctx->eng->geometry(nx, ny, nz, info);
  return ctx->eng->plan(nx, ny, nz, info);
}

int mc3_host_alloc(size_t bytes, void** ptr) {
  if (!ptr || bytes == 0) return MC3_EINVAL;
  *ptr = nullptr;
  if (cudaHostAlloc(ptr, bytes, cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    *ptr = nullptr;
    return MC3_ENOMEM;
  }
  return MC3_OK;
}

int mc3_host_free(void* ptr) {
  if (!ptr) return MC3_OK;
  return cudaFreeHost(ptr) == cudaSuccess ? MC3_OK : MC3_ECUDA;
}

int mc3_set_dark(mc3_ctx* ctx, const float* dark, int nx, int ny, int on_device) {
  if (!ctx) return MC3_EINVAL;
  return ctx->eng->set_dark(dark, nx, ny, on_device != 0);
}

int mc3_set_defects(mc3_ctx* ctx, const unsigned char* mask, int nx, int ny) {
  if (!ctx) return MC3_EINVAL;
  return ctx->eng->set_defects(mask, nx, ny);
}

int mc3_set_gain(mc3_ctx* ctx, const float* gain, int nx, int ny, int on_device) {
  if (!ctx) return MC3_EINVAL;
  return ctx->eng->set_gain(gain, nx, ny, on_device != 0);
}

namespace {
// Movies still queued: the context belongs to its worker thread.
bool queue_busy(mc3_ctx* ctx) { return ctx->queue && ctx->queue->outstanding() > 0; }
}  // namespace

int mc3_process_movie(mc3_ctx* ctx, const mc3_movie* movie, mc3_result* out) {
  if (!ctx || !movie || queue_busy(ctx)) return MC3_EINVAL;
  return ctx->eng->process(*movie, out);
}

int mc3_submit(mc3_ctx* ctx, const mc3_movie* movie, mc3_result* out, int* ticket) {
  if (!ctx || !movie || !ticket || !movie->frames) return MC3_EINVAL;
  if (!ctx->queue) {
    ctx->queue = new (std::nothrow) MovieQueue(ctx->eng);
    if (!ctx->queue) return MC3_ENOMEM;
  }
  return ctx->queue->submit(*movie, out, ticket);
}

int mc3_autotune(mc3_ctx* ctx, int nx, int ny, int nz, const char* json_path, double* ms_best) {
  if (!ctx || nx < 16 || ny < 16 || nz < 3 || queue_busy(ctx)) return MC3_EINVAL;
  TuningEntry e;
  int s = ctx->eng->autotune(nx, ny, nz, &e);
  if (s != kOk) return s;
  if (ms_best) *ms_best = e.best_ms;
  if (json_path) {
    // the file keeps the entries of other sizes; this size's entry is replaced
    std::vector<TuningEntry> all;
    if (FILE* f = std::fopen(json_path, "rb")) {
      std::string text;
      char buf[4096];
      size_t n;
      while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
      std::fclose(f);
      parse_tuning_json(text, &all);
    }
    for (auto it = all.begin(); it != all.end();)
      it = (it->nx == e.nx && it->ny == e.ny && it->nz == e.nz && it->px == e.px && it->py == e.py)
               ? all.erase(it)
               : it + 1;
    all.push_back(e);
    cudaDeviceProp prop;
    const char* dev = cudaGetDeviceProperties(&prop, ctx->eng->device) == cudaSuccess ? prop.name : "";
    const std::string js = tuning_json(all, dev);
    FILE* f = std::fopen(json_path, "wb");
    if (!f) return MC3_EIO;
    const bool ok = std::fwrite(js.data(), 1, js.size(), f) == js.size();
    std::fclose(f);
    if (!ok) return MC3_EIO;
  }
  return MC3_OK;
}

int mc3_load_tuning(mc3_ctx* ctx, const char* json_path) {
  if (!ctx || !json_path || queue_busy(ctx)) return MC3_EINVAL;
  FILE* f = std::fopen(json_path, "rb");
  if (!f) return MC3_EIO;
  std::string text;
  char buf[4096];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
  std::fclose(f);
  std::vector<TuningEntry> all;
  if (parse_tuning_json(text, &all) != 0) return MC3_EIO;
  for (const TuningEntry& e : all) {
    auto& tab = ctx->eng->tuning_table;
    for (auto it = tab.begin(); it != tab.end();)
      it = (it->nx == e.nx && it->ny == e.ny && it->nz == e.nz && it->px == e.px && it->py == e.py)
               ? tab.erase(it)
               : it + 1;
    tab.push_back(e);
  }
  return MC3_OK;
}

int mc3_wait(mc3_ctx* ctx, int ticket, double* latency_ms) {
  if (!ctx || !ctx->queue) return MC3_EINVAL;
  return ctx->queue->wait(ticket, latency_ms);
}

int mc3_estimate_ctf(mc3_ctx* ctx, const float* image, int nx, int ny, int on_device, float pix_size,
                     float kv, float cs, float amp_cont, float ext_phase, float* result6,
                     float* spectrum512) {
  if (!ctx || !image || !result6 || nx < 2 || ny < 2 || !(pix_size > 0) || !(kv > 0) ||
      !(amp_cont >= 0 && amp_cont < 1))
    return MC3_EINVAL;
  Engine* e = ctx->eng;
  MC3_CUDA(cudaSetDevice(e->device));
  const float* d_img = image;
  if (!on_device) {
    MC3_TRY(e->d_out.ensure(sizeof(float) * (size_t)nx * ny));
    MC3_CUDA(cudaMemcpyAsync(e->d_out.p, image, sizeof(float) * (size_t)nx * ny, cudaMemcpyHostToDevice,
                             e->stream));
    d_img = e->d_out.as<float>();
  }
  return estimate_ctf(d_img, nx, ny, pix_size, kv, cs, amp_cont, ext_phase, result6, spectrum512,
                      on_device != 0, e->ctf, e->stream);
}

int mc3_prefetch_movie(mc3_ctx* ctx, const mc3_movie* movie) {
  if (!ctx || !movie || queue_busy(ctx)) return MC3_EINVAL;
  return ctx->eng->prefetch(*movie);
}

int mc3_proposal_create(const int* spec, int n_layers, int nout, unsigned seed, int gpu,
                        mc3_proposal** out) {
  if (!spec || !out || n_layers < 1 || nout < 1 || spec[0] != 2) return MC3_EINVAL;
  *out = nullptr;
  if (cudaSetDevice(gpu) != cudaSuccess) {
    cudaGetLastError();
    return MC3_ECUDA;
  }
  mc3_proposal* p = new (std::nothrow) mc3_proposal;
  if (!p) return MC3_ENOMEM;
  p->gpu = gpu;
  const int s = p->net.create(std::vector<int>(spec, spec + 5 * n_layers), nout, seed);
  if (s != kOk) {
    delete p;
    return s;
  }
  *out = p;
  return MC3_OK;
}

int mc3_proposal_destroy(mc3_proposal* p) {
  if (!p) return MC3_EINVAL;
  cudaSetDevice(p->gpu);
  delete p;
  return MC3_OK;
}

int mc3_proposal_num_params(mc3_proposal* p, long* n) {
  if (!p || !n) return MC3_EINVAL;
  *n = p->net.nparams;
  return MC3_OK;
}

int mc3_proposal_get_params(mc3_proposal* p, float* params) {
  if (!p || !params) return MC3_EINVAL;
  MC3_CUDA(cudaSetDevice(p->gpu));
  MC3_CUDA(cudaMemcpy(params, p->net.d_params, sizeof(float) * p->net.nparams, cudaMemcpyDeviceToHost));
  return MC3_OK;
}

int mc3_proposal_set_params(mc3_proposal* p, const float* params) {
  if (!p || !params) return MC3_EINVAL;
  MC3_CUDA(cudaSetDevice(p->gpu));
  MC3_CUDA(cudaMemcpy(p->net.d_params, params, sizeof(float) * p->net.nparams, cudaMemcpyHostToDevice));
  return MC3_OK;
}

namespace {
// Batch inputs on the device: the caller's pointers, or copies into the net's buffers.
int proposal_inputs(mc3_proposal* p, const float* x, const float* target, int batch, int h, int w,
                    int on_device, const float** dx, const float** dt, cudaStream_t st) {
  MC3_TRY(p->net.ensure(batch, h, w, st));
  if (on_device) {
    *dx = x;
    *dt = target;
    return kOk;
  }
  const size_t nx = (size_t)batch * 2 * h * w;
  MC3_CUDA(cudaMemcpyAsync(p->net.d_x, x, sizeof(float) * nx, cudaMemcpyHostToDevice, st));
  *dx = p->net.d_x;
  *dt = nullptr;
  if (target) {
    MC3_CUDA(cudaMemcpyAsync(p->net.d_target, target, sizeof(float) * batch * p->net.nout,
                             cudaMemcpyHostToDevice, st));
    *dt = p->net.d_target;
  }
  return kOk;
}

double batch_loss(mc3_proposal* p, int batch, int* status) {
  std::vector<float> l(batch);
  *status = cudaMemcpy(l.data(), p->net.d_loss, sizeof(float) * batch, cudaMemcpyDeviceToHost) ==
                    cudaSuccess
                ? kOk
                : kECuda;
  double s = 0.0;
  for (float v : l) s += v;
  return s;
}
}  // namespace

int mc3_proposal_loss_grad(mc3_proposal* p, const float* x, int batch, int h, int w,
                           const float* target, double* loss, float* grad, float* out) {
  if (!p || !x || !target || batch < 1 || h < 1 || w < 1) return MC3_EINVAL;
  MC3_CUDA(cudaSetDevice(p->gpu));
  cudaStream_t st = nullptr;
  const float *dx, *dt;
  MC3_TRY(proposal_inputs(p, x, target, batch, h, w, 0, &dx, &dt, st));
  MC3_TRY(p->net.run(dx, batch, h, w, dt, st));
  MC3_CUDA(cudaStreamSynchronize(st));
  int s = kOk;
  const double l = batch_loss(p, batch, &s);
  if (s) return s;
  if (loss) *loss = l;
  if (grad)
    MC3_CUDA(cudaMemcpy(grad, p->net.d_grad, sizeof(float) * p->net.nparams, cudaMemcpyDeviceToHost));
  if (out)
    MC3_CUDA(cudaMemcpy(out, p->net.d_out, sizeof(float) * batch * p->net.nout, cudaMemcpyDeviceToHost));
  return MC3_OK;
}

int mc3_proposal_train_step(mc3_proposal* p, const float* x, const float* target, int batch,
                            int h, int w, int on_device, float lr, double* loss) {
  if (!p || !x || !target || batch < 1 || h < 1 || w < 1 || !(lr > 0)) return MC3_EINVAL;
  MC3_CUDA(cudaSetDevice(p->gpu));
  cudaStream_t st = nullptr;
  const float *dx, *dt;
  MC3_TRY(proposal_inputs(p, x, target, batch, h, w, on_device, &dx, &dt, st));
  MC3_TRY(p->net.run(dx, batch, h, w, dt, st));
  MC3_TRY(p->net.adam_step(batch, lr, st));
  MC3_CUDA(cudaStreamSynchronize(st));
  int s = kOk;
  const double l = batch_loss(p, batch, &s);
  if (s) return s;
  if (loss) *loss = l / batch;
  return MC3_OK;
}

int mc3_proposal_predict(mc3_proposal* p, const float* x, int batch, int h, int w, int on_device,
                         float* out) {
  if (!p || !x || !out || batch < 1 || h < 1 || w < 1) return MC3_EINVAL;
  MC3_CUDA(cudaSetDevice(p->gpu));
  cudaStream_t st = nullptr;
  const float *dx, *dt;
  MC3_TRY(proposal_inputs(p, x, nullptr, batch, h, w, on_device, &dx, &dt, st));
  MC3_TRY(p->net.run(dx, batch, h, w, nullptr, st));
  MC3_CUDA(cudaMemcpy(out, p->net.d_out, sizeof(float) * batch * p->net.nout, cudaMemcpyDeviceToHost));
  return MC3_OK;
}

int mc3_proposal_pair_inputs(const float* frames, int nx, int ny, int nz, const int* pairs, int n,
                             int bin, float* x, void* stream) {
  if (!frames || !pairs || !x || n < 1 || nz < 1 || bin < 1 || nx / bin < 1 || ny / bin < 1)
    return MC3_EINVAL;
  for (int i = 0; i < 2 * n; ++i)
    if (pairs[i] < 0 || pairs[i] >= nz) return MC3_EINVAL;
  cudaStream_t st = as_stream(stream);
  int* d = nullptr;
  MC3_CUDA(cudaMalloc(&d, sizeof(int) * 2 * n));
  int s = cudaMemcpyAsync(d, pairs, sizeof(int) * 2 * n, cudaMemcpyHostToDevice, st) == cudaSuccess
              ? kOk
              : kECuda;
  if (s == kOk) s = proposal::pair_inputs(frames, nx, ny, (long)nx * ny, d, n, bin, x, st);
  if (s == kOk && cudaStreamSynchronize(st) != cudaSuccess) s = kECuda;
  cudaFree(d);
  return s;
}

int mc3_set_first_iterate(mc3_ctx* ctx, const float* global_xy, int nz, int max_iter) {
  if (!ctx || queue_busy(ctx)) return MC3_EINVAL;
  if (!global_xy) {
    ctx->eng->first_iterate.clear();
    return MC3_OK;
  }
  if (nz < 1) return MC3_EINVAL;
  ctx->eng->first_iterate.assign(global_xy, global_xy + 2 * (size_t)nz);
  ctx->eng->first_iterate_max = max_iter > 0 ? max_iter : 3;
  return MC3_OK;
}

int mc3_set_patch_centers(mc3_ctx* ctx, const float* centers_xy, int n_patches) {
  if (!ctx || queue_busy(ctx)) return MC3_EINVAL;
  if (!centers_xy) {
    ctx->eng->patch_centers_given.clear();
    return MC3_OK;
  }
  if (n_patches < 1) return MC3_EINVAL;
  for (int i = 0; i < 2 * n_patches; ++i)  // finite pixel coordinates
    if (!std::isfinite(centers_xy[i]) || std::fabs(centers_xy[i]) > 1.0e6f) return MC3_EINVAL;
  ctx->eng->patch_centers_given.assign(centers_xy, centers_xy + 2 * (size_t)n_patches);
  return MC3_OK;
}

int mc3_set_alignment(mc3_ctx* ctx, const mc3_alignment* aln) {
  if (!ctx) return MC3_EINVAL;
  return ctx->eng->set_alignment(aln);
}

int mc3_set_frame_integration(mc3_ctx* ctx, const mc3_frame_integration* fi) {
  if (!ctx) return MC3_EINVAL;
  return ctx->eng->set_frame_integration(fi);
}

int mc3_read_fmint_file(const char* path, float fm_dose, int max_entries, int* group_size,
                        int* int_size, float* dose, int* n_entries) {
  if (!path || !n_entries || max_entries < 0) return MC3_EINVAL;
  std::vector<int> g, n;
  std::vector<float> d;
  if (!host::read_fmint_file(path, fm_dose, g, n, d)) return MC3_EIO;
  *n_entries = (int)g.size();
  for (int i = 0; i < (int)g.size() && i < max_entries; ++i) {
    if (group_size) group_size[i] = g[i];
    if (int_size) int_size[i] = n[i];
    if (dose) dose[i] = d[i];
  }
  return MC3_OK;
}

int mc3_frame_groups(const int* start, const int* size, int n, int bin_z, int max_groups,
                     int* n_groups, int* g_start, int* g_size, float* g_center) {
  if (!start || !size || n < 1 || bin_z < 1 || !n_groups) return MC3_EINVAL;
  host::FmInt t;
  t.start.assign(start, start + n);
  t.size.assign(size, size + n);
  t.dose.assign(n, 0.0f);
  t.acc.assign(n, 0.0f);
  t.centers();
  host::FrameGroups g;
  g.setup(t, bin_z);
  *n_groups = g.count();
  for (int i = 0; i < g.count() && i < max_groups; ++i) {
    if (g_start) g_start[i] = g.start[i];
    if (g_size) g_size[i] = g.size[i];
    if (g_center) g_center[i] = g.center[i];
  }
  return MC3_OK;
}

int mc3_frame_integration_tables(const int* group_size, const int* int_size, const float* dose,
                                 int n_entries, int n_raw, float fm_dose, int throw_first,
                                 int throw_last, int max_int, int* n_int, int* start, int* size,
                                 float* acc_dose, int* dose_weight) {
  if (n_raw < 1 || n_entries < 0 || !n_int || throw_first < 0 || throw_last < 0) return MC3_EINVAL;
  if (n_entries > 0 && (!group_size || !int_size || !dose)) return MC3_EINVAL;
  for (int i = 0; i < n_entries; ++i)
    if (int_size[i] < 1 || group_size[i] < 0) return MC3_EINVAL;
  // CReadFmIntFile::NeedIntegrate (DataUtil/CReadFmIntFile.cpp:73-89)
  bool integrate = false;
  if (n_entries > 0 && std::fabs(dose[0] - dose[n_entries - 1]) < 0.0001f)
    for (int i = 0; i < n_entries; ++i) integrate = integrate || int_size[i] > 1;
  host::FmInt t;
  if (integrate) {
    t.integrate(std::vector<int>(group_size, group_size + n_entries),
                std::vector<int>(int_size, int_size + n_entries), dose[0], n_raw);
    t.drop(throw_first, throw_last);  // mThrowIntFrames (:231-256)
  } else {
    // CFmIntParam::mSetup (:118-136): the kept raw frames, doses counted from 1
    const int keep = n_raw - throw_first - throw_last;
    if (keep < 1) return MC3_EINVAL;
    t.plain(keep, fm_dose);
    for (int& st : t.start) st += throw_first;
    t.centers();
  }
  *n_int = t.count();
  for (int i = 0; i < t.count() && i < max_int; ++i) {
    if (start) start[i] = t.start[i];
    if (size) size[i] = t.size[i];
    if (acc_dose) acc_dose[i] = t.acc[i];
  }
  if (dose_weight) *dose_weight = (n_entries > 0 && dose[0] > 0) ? 1 : 0;  // HasDose
  return MC3_OK;
}

// ---- components ----
int mc3_rfft_rows(const float* in, int in_pitch, float* out, int out_pitch, int nx, int n_rows,
                  int method, void* stream) {
  if (!in || !out || nx < 2 || (nx & 1) || n_rows < 1 || in_pitch < nx ||
      out_pitch < nx / 2 + 1 || (method != 0 && method != 1))
    return MC3_EINVAL;
  cudaStream_t st = as_stream(stream);
  Batch b{1, 1, 0, nullptr, 0};
  int s = method == 1 ? dft_rows_r2c(in, in_pitch, reinterpret_cast<float2*>(out), out_pitch, nx,
                                     n_rows, b, 1.0f, st)
                      : row_r2c(in, in_pitch, reinterpret_cast<float2*>(out), out_pitch, nx,
                                n_rows, b, 1.0f, st);
  if (s) return s;
  if (cudaStreamSynchronize(st) != cudaSuccess) return MC3_ECUDA;
  if (method == 1) {
    int flag = 0;
    s = dft_gemm_error(true, &flag);
    if (s) return s;
    if (flag) return MC3_ETIMEOUT;
  }
  return MC3_OK;
}

int mc3_fft_forward(float* frames, int nx, int ny, int nz, int normalise, void* stream) {
  if (!frames || nx < 2 || (nx & 1) || ny < 1 || nz < 1) return MC3_EINVAL;
  const int cmpX = nx / 2 + 1;
  const long ncmp = (long)cmpX * ny;
  cudaStream_t st = as_stream(stream);
  Batch b{nz, nz, ncmp * 2, nullptr, ncmp};
  int s = row_r2c(frames, 2 * cmpX, reinterpret_cast<float2*>(frames), cmpX, nx, ny, b, 1.0f, st);
  if (s) return s;
  Batch bc{nz, nz, ncmp, nullptr, ncmp};
  ColOps ops{};
  ops.dir = -1;
  ops.scale = normalise ? (float)(1.0 / nx / ny) : 1.0f;
  float2* c = reinterpret_cast<float2*>(frames);
  return col_fft(c, c, cmpX, cmpX, ny, bc, ops, st);
}

int mc3_fft_inverse(float* frames, int nx, int ny, int nz, void* stream) {
  if (!frames || nx < 2 || (nx & 1) || ny < 1 || nz < 1) return MC3_EINVAL;
  const int cmpX = nx / 2 + 1;
  const long ncmp = (long)cmpX * ny;
  cudaStream_t st = as_stream(stream);
  float2* c = reinterpret_cast<float2*>(frames);
  Batch bc{nz, nz, ncmp, nullptr, ncmp};
  ColOps ops{};
  ops.dir = 1;
  ops.scale = 1.0f;
  int s = col_fft(c, c, cmpX, cmpX, ny, bc, ops, st);
  if (s) return s;
  Batch br{nz, nz, ncmp, nullptr, ncmp * 2};
  return row_c2r(c, cmpX, frames, 2 * cmpX, nx, ny, br, st);
}

int mc3_fourier_crop(const float* in, int in_cmp_x, int in_cmp_y, float* out, int out_cmp_x,
                     int out_cmp_y, void* stream) {
  if (!in || !out || out_cmp_x > in_cmp_x || out_cmp_y > in_cmp_y) return MC3_EINVAL;
  return fourier_crop(reinterpret_cast<const float2*>(in), in_cmp_x, in_cmp_y,
                      reinterpret_cast<float2*>(out), out_cmp_x, out_cmp_y, as_stream(stream));
}

int mc3_detect_bad_pixels(const float* sum, int nx, int ny, unsigned char* bad, void* stream) {
  if (!sum || !bad || nx < 8 || ny < 8 || (nx & 1)) return MC3_EINVAL;
  const long pad = 2 * (nx / 2 + 1);
  float *cc = nullptr, *part = nullptr, *mom = nullptr;
  if (cudaMalloc(&cc, sizeof(float) * pad * ny) != cudaSuccess) return MC3_ENOMEM;
  if (cudaMalloc(&part, sizeof(float) * 1024) != cudaSuccess) { cudaFree(cc); return MC3_ENOMEM; }
  if (cudaMalloc(&mom, sizeof(float) * 16) != cudaSuccess) { cudaFree(cc); cudaFree(part); return MC3_ENOMEM; }
  float tpl[36];
  host::defect_template(6, tpl);
  cudaStream_t st = as_stream(stream);
  int s = detect_bad_pixels(sum, nx, ny, cc, part, mom, bad, tpl, 6, st);
  if (s == kOk && cudaStreamSynchronize(st) != cudaSuccess) s = MC3_ECUDA;
  cudaFree(cc);
  cudaFree(part);
  cudaFree(mom);
  return s;
}

int mc3_correct_bad_pixels(float* frames, int nx, int ny, int nz, const unsigned char* bad,
                           void* stream) {
  if (!frames || !bad || nx < 2 || (nx & 1) || ny < 1 || nz < 1) return MC3_EINVAL;
  const long pad = 2 * (nx / 2 + 1);
  int* cnt = nullptr;
  int2* list = nullptr;
  if (cudaMalloc(&cnt, sizeof(int)) != cudaSuccess) return MC3_ENOMEM;
  if (cudaMalloc(&list, sizeof(int2) * (size_t)nx * ny) != cudaSuccess) {
    cudaFree(cnt);
    return MC3_ENOMEM;
  }
  cudaStream_t st = as_stream(stream);
  int s = correct_bad_pixels(frames, pad * ny, nz, bad, nx, ny, cnt, list, st);
  if (s == kOk && cudaStreamSynchronize(st) != cudaSuccess) s = MC3_ECUDA;
  cudaFree(cnt);
  cudaFree(list);
  return s;
}

int mc3_local_gather(const float* in, float* out, int nx, int ny, const float* centers,
                     const float* shifts, const unsigned char* bad, int n_patches, void* stream) {
  if (!in || !out || !centers || !shifts || n_patches < 1) return MC3_EINVAL;
  const long pad = 2 * (nx / 2 + 1);
  return local_gather(in, pad * ny, out, pad * ny, 1, nx, ny, centers,
                      reinterpret_cast<const float2*>(shifts), nullptr, bad, nullptr, n_patches,
                      as_stream(stream));
}

int mc3_phase_shift(const float* in, float* out, int cmp_x, int cmp_y, float sx, float sy,
                    int accumulate, void* stream) {
  if (!in || !out || cmp_x < 2 || cmp_y < 1) return MC3_EINVAL;
  cudaStream_t st = as_stream(stream);
  float2 *sh = nullptr, *ex = nullptr, *ey = nullptr;
  int s = MC3_OK;
  if (cudaMalloc(&sh, sizeof(float2)) != cudaSuccess || cudaMalloc(&ex, sizeof(float2) * cmp_x) != cudaSuccess ||
      cudaMalloc(&ey, sizeof(float2) * cmp_y) != cudaSuccess) {
    s = MC3_ENOMEM;
  }
  if (s == MC3_OK) {
    float2 h;
    h.x = sx;
    h.y = sy;
    if (cudaMemcpyAsync(sh, &h, sizeof(float2), cudaMemcpyHostToDevice, st) != cudaSuccess) s = MC3_ECUDA;
    if (s == MC3_OK) s = phase_tables(sh, 1, cmp_x, cmp_y, ex, ey, false, st);
    if (s == MC3_OK)
      s = phase_apply(reinterpret_cast<const float2*>(in), reinterpret_cast<float2*>(out), cmp_x, cmp_y,
                      ex, ey, accumulate != 0, st);
    if (s == MC3_OK && cudaStreamSynchronize(st) != cudaSuccess) s = MC3_ECUDA;
  }
  cudaFree(sh);
  cudaFree(ex);
  cudaFree(ey);
  return s;
}

int mc3_correlate(const float* group, const float* sum, int cmp_x, int cmp_y, float bfactor,
                  int phase_only, int sea_x, int sea_y, float* window, float* shift_host,
                  void* stream) {
  if (!group || !sum || cmp_x < 3 || cmp_y < 4 || sea_x < 3 || sea_y < 3) return MC3_EINVAL;
  if (sea_x > (cmp_x - 1) * 2 || sea_y > cmp_y) return MC3_EINVAL;
  cudaStream_t st = as_stream(stream);
  // Treat `group` as a one-frame stack whose single group is that frame;
  // corr_cols computes conj(G) (S - G) with S = `sum`.
  const size_t nel = (size_t)cmp_x * cmp_y;
  float2 *sh = nullptr, *ex = nullptr, *ey = nullptr, *T = nullptr, *pk = nullptr;
  int *act = nullptr, *gs = nullptr, *gz = nullptr;
  float* win = nullptr;
  int s = MC3_OK;
  if (cudaMalloc(&sh, sizeof(float2)) != cudaSuccess || cudaMalloc(&ex, sizeof(float2) * cmp_x) != cudaSuccess ||
      cudaMalloc(&ey, sizeof(float2) * cmp_y) != cudaSuccess || cudaMalloc(&act, sizeof(int) * 3) != cudaSuccess ||
      cudaMalloc(&T, sizeof(float2) * (size_t)sea_y * cmp_x) != cudaSuccess ||
      cudaMalloc(&win, sizeof(float) * (size_t)sea_x * sea_y) != cudaSuccess ||
      cudaMalloc(&pk, sizeof(float2)) != cudaSuccess) {
    s = MC3_ENOMEM;
  }
  gs = act + 1;
  gz = act + 2;
  if (s == MC3_OK) {
    float2 h;
    h.x = 0.f;
    h.y = 0.f;
    int hi[3] = {0, 0, 1};
    cudaMemcpyAsync(sh, &h, sizeof(float2), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(act, hi, sizeof(int) * 3, cudaMemcpyHostToDevice, st);
    s = phase_tables(sh, 1, cmp_x, cmp_y, ex, ey, false, st);
    AlignDims d{};
    d.cmpX = cmp_x;
    d.cmpY = cmp_y;
    d.N = 1;
    d.stack_stride = (long)nel;
    d.G = 1;
    d.seaX = sea_x;
    d.seaY = sea_y;
    d.A = 1;
    if (s == MC3_OK)
      s = corr_cols(reinterpret_cast<const float2*>(group), act, ex, ey,
                    reinterpret_cast<const float2*>(sum), gs, gz, bfactor, phase_only, T, d, st);
    if (s == MC3_OK) s = corr_rows(T, win, d, st);
    if (s == MC3_OK) s = peak_search(win, pk, d, st);
    if (s == MC3_OK && window)
      cudaMemcpyAsync(window, win, sizeof(float) * sea_x * sea_y, cudaMemcpyDeviceToDevice, st);
    float2 r;
    if (s == MC3_OK) {
      cudaMemcpyAsync(&r, pk, sizeof(float2), cudaMemcpyDeviceToHost, st);
      if (cudaStreamSynchronize(st) != cudaSuccess) s = MC3_ECUDA;
      if (s == MC3_OK && shift_host) {
        shift_host[0] = r.x;
        shift_host[1] = r.y;
      }
    }
  }
  cudaFree(sh);
  cudaFree(ex);
  cudaFree(ey);
  cudaFree(act);
  cudaFree(T);
  cudaFree(win);
  cudaFree(pk);
  return s;
}

int mc3_iterative_align(mc3_ctx* ctx, const float* stack, int cmp_x, int cmp_y, int n, int group,
                        int max_iter, float tol, float bfactor, int phase_only, float* shifts_host,
                        int* iters) {
  if (!ctx || !stack || !shifts_host || n < 3 || group < 1 || max_iter < 1) return MC3_EINVAL;
  Engine* e = ctx->eng;
  const int saved_iter = e->prm.iter, saved_po = e->prm.phase_only;
  e->prm.iter = max_iter;
  e->prm.phase_only = phase_only;
  host::FrameGroups g;
  g.setup(n, group);
  std::vector<host::StackShift> sh;
  std::vector<int> it;
  std::vector<std::vector<float>> err;
  int s = e->align_stacks(reinterpret_cast<const float2*>(stack), (long)cmp_x * cmp_y * n, 1, cmp_x,
                          cmp_y, n, g, bfactor, tol, sh, it, err);
  e->prm.iter = saved_iter;
  e->prm.phase_only = saved_po;
  if (s != kOk) return s;
  for (int f = 0; f < n; ++f) {
    shifts_host[2 * f] = sh[0].x(f);
    shifts_host[2 * f + 1] = sh[0].y(f);
  }
  if (iters) *iters = it[0];
  return MC3_OK;
}

int mc3_dose_weighted_sums(mc3_ctx* ctx, const float* spectra, int nx, int ny, int nz,
                           const float* shifts_host, float* sums, int* n_sums) {
  if (!ctx || !spectra || !sums || !shifts_host) return MC3_EINVAL;
  Engine* e = ctx->eng;
  Geometry g;
  int s = g.compute(nx, ny, nz, e->prm);
  if (s) return s;
  host::StackShift fs;
  fs.setup(nz);
  for (int f = 0; f < nz; ++f) {
    fs.x(f) = shifts_host[2 * f];
    fs.y(f) = shifts_host[2 * f + 1];
  }
  const size_t ncmp = (size_t)g.cmpX * g.cmpY;
  cudaStream_t st = e->stream;
  if ((s = e->d_acc.ensure(sizeof(float) * nz)) || (s = e->d_Wn.ensure(sizeof(float) * ncmp))) return s;
  std::vector<float> acc(nz);
  for (int i = 0; i < nz; ++i) acc[i] = e->prm.fm_dose * (i + 1);
  if (cudaMemcpyAsync(e->d_acc.p, acc.data(), sizeof(float) * nz, cudaMemcpyHostToDevice, st) != cudaSuccess)
    return MC3_ECUDA;
  DoseParams dp{};
  dp.enabled = g.dw ? 1 : 0;
  dp.dws = g.dws ? 1 : 0;
  dp.pix_size = e->prm.pix_size;
  dp.kv_factor = host::kv_factor(e->prm.kv);
  dp.sum_range[0] = e->prm.sum_range[0];
  dp.sum_range[1] = e->prm.sum_range[1];
  dp.split = e->prm.split_sum ? 1 : 0;
  e->wn_valid = false;  // d_Wn is rebuilt here for this call's geometry
  if (g.dw && (s = dose_norm(e->d_acc.as<float>(), nz, g.cmpX, g.cmpY, dp.pix_size, dp.kv_factor,
                             e->d_Wn.as<float>(), st)))
    return s;
  if ((s = e->global_sums(reinterpret_cast<const float2*>(spectra), nz, fs, g))) return s;
  s = frame_sums(reinterpret_cast<const float2*>(spectra), (long)ncmp, nz, g.cmpX, g.cmpY,
                 e->d_fex.as<float2>(), e->d_fey.as<float2>(), e->d_acc.as<float>(), e->d_Wn.as<float>(),
                 dp, reinterpret_cast<float2*>(sums), g.nSums, st);
  if (s) return s;
  if (cudaStreamSynchronize(st) != cudaSuccess) return MC3_ECUDA;
  if (n_sums) *n_sums = g.nSums;
  return MC3_OK;
}

// ---- diagnostics ----
void mc3_profile_enable(int on) { prof::enable(on != 0); }

int mc3_profile_read(char* buf, size_t len, int reset) {
  if (!buf || len == 0) return MC3_EINVAL;
  std::string s = prof::json();
  if (reset) prof::reset();
  if (s.size() + 1 > len) return MC3_EINVAL;
  std::memcpy(buf, s.c_str(), s.size() + 1);
  return MC3_OK;
}

unsigned long long mc3_kernel_launches(void) { return prof::launches(); }

// ---- host bookkeeping ----
void mc3_peak2d(const float* window, int sea_x, int sea_y, float* shift) {
  host::peak2d(window, sea_x, sea_y, shift);
}

void mc3_remove_spikes(float* sx, float* sy, int n) { host::remove_spikes(sx, sy, n); }

int mc3_lin_eqs(float* coeff, float* vals, int dim) { return host::lin_eqs(coeff, vals, dim) ? 1 : 0; }

void mc3_smooth_shifts(float* sx, float* sy, int n, float weight) {
  host::StackShift s;
  s.setup(n);
  std::memcpy(s.v.data(), sx, sizeof(float) * n);
  std::memcpy(s.v.data() + n, sy, sizeof(float) * n);
  s.smooth(weight);
  std::memcpy(sx, s.v.data(), sizeof(float) * n);
  std::memcpy(sy, s.v.data() + n, sizeof(float) * n);
}

void mc3_patch_make_relative(float* shifts, int nz, int n_patches) {
  std::vector<float> v(shifts, shifts + (size_t)nz * n_patches * 2);
  host::patch_make_relative(v, nz, n_patches);
  std::memcpy(shifts, v.data(), sizeof(float) * v.size());
}

void mc3_patch_detect_bads(const float* shifts, const float* centers, int nz, int n_patches,
                           int nx, int ny, unsigned char* bad) {
  host::patch_detect_bads(shifts, centers, nz, n_patches, nx, ny, bad);
}

int mc3_patch_starts_from_centers(const float* centers, int n_patches, float bin_x, float bin_y,
                                  int xcf_x, int xcf_y, int pat_x, int pat_y, int* starts) {
  if (!centers || !starts || n_patches < 1 || !(bin_x > 0.0f) || !(bin_y > 0.0f) ||
      pat_x < 1 || pat_y < 1 || pat_x > xcf_x || pat_y > xcf_y)
    return MC3_EINVAL;
  for (int i = 0; i < 2 * n_patches; ++i)
    if (!std::isfinite(centers[i]) || std::fabs(centers[i]) > 1.0e6f) return MC3_EINVAL;
  std::vector<int> s;
  host::patch_starts_from_centers(centers, n_patches, bin_x, bin_y, xcf_x, xcf_y, pat_x, pat_y, s);
  std::memcpy(starts, s.data(), sizeof(int) * s.size());
  return MC3_OK;
}

}  // extern "C"
