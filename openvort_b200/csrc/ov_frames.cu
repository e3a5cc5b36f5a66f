// ov_frames.cu - frame output and input.
//
// Text frames are the reference's save_tangle files (src/vortex_utils.c:
// 308-345), byte for byte: one line per node in its traversal order, the
// numbers printed with the same printf formats.  The formatting is split
// over host threads by rows; the rows are written in order.
//
// Binary frames carry what a restart needs and the text format lacks: the
// simulation time (the reference's README lists its absence as a known
// issue) and every slot's arrays as they are, EMPTY slots included.
//
// From a device-resident state (ov_state_save_frame) a frame is taken
// without stopping the state: device-to-device copies of its arrays on the
// state's stream, then a copy into pinned host memory on a separate stream,
// then a writer thread formats and writes the file while the state steps
// on.  ov_frame_wait waits for the writes.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ov_internal.h"

namespace {

// slot arrays in host memory
struct FrameView {
  int n = 0;
  const double* pos = nullptr;
  const double* vels = nullptr;
  const double* tan = nullptr;
  const double* nrm = nullptr;
  const double* dxi = nullptr;
  const int* links = nullptr;    // (forward, reverse) per slot
  const int* status = nullptr;   // (status, pin_wall) per slot
};

FrameView view_of(const tangle_state* t) {
  FrameView v;
  v.n = t->N;
  v.pos = &t->vnodes[0].p[0];
  v.vels = t->vels ? &t->vels[0].p[0] : nullptr;
  v.tan = t->tangents ? &t->tangents[0].p[0] : nullptr;
  v.nrm = t->normals ? &t->normals[0].p[0] : nullptr;
  v.dxi = t->dxi;
  v.links = reinterpret_cast<const int*>(t->connections);
  v.status = reinterpret_cast<const int*>(t->status);
  return v;
}

struct Row {
  int vortex, slot;
};

// save_tangle's traversal (src/vortex_utils.c:308-345): for each slot k not
// yet visited and not EMPTY, its vortex: forward from k until the next node
// is k again; at an open end, from k's reverse neighbour backwards while
// that node's reverse link is above 0.  The reference's tests treat slot 0
// as "no node" on the way back and after the walk (curr > 0), and they are
// kept as they are.  Walks are bounded by the slot count (a link cycle that
// does not return to k is an error).
bool frame_order(const FrameView& v, std::vector<Row>& rows) {
  const int n = v.n;
  auto fwd = [&](int k) { return v.links[2 * k]; };
  auto rev = [&](int k) { return v.links[2 * k + 1]; };
  std::vector<char> visited(n, 0);
  rows.clear();
  rows.reserve(n);
  int vidx = 0;
  for (int k = 0; k < n; ++k) {
    if (visited[k]) continue;
    if (v.status[2 * k] == EMPTY) {
      visited[k] = 1;
      continue;
    }
    const int first = k;
    int curr = k;
    long steps = 0;
    while (fwd(curr) != first) {
      rows.push_back({vidx, curr});
      visited[curr] = 1;
      curr = fwd(curr);
      if (++steps > n || curr >= n) return false;
      if (curr < 0) {
        curr = rev(first);
        while (curr > 0 && rev(curr) > 0) {
          rows.push_back({vidx, curr});
          visited[curr] = 1;
          curr = rev(curr);
          if (++steps > n || curr >= n) return false;
        }
        break;
      }
    }
    if (curr > 0) {
      rows.push_back({vidx, curr});
      visited[curr] = 1;
    }
    ++vidx;
  }
  return true;
}

// one line of save_point (src/vortex_utils.c:271-286)
void format_row(const FrameView& v, const Row& r, std::string& out) {
  char buf[1024];
  const int i = r.slot;
  const double* p = v.pos + 3 * (size_t)i;
  const double* u = v.vels + 3 * (size_t)i;
  const double* t = v.tan + 3 * (size_t)i;
  const double* m = v.nrm + 3 * (size_t)i;
  const int len = snprintf(buf, sizeof(buf),
                           "%d\t%.15g\t%.15g\t%.15g\t%.15g\t%.15g\t%.15g\t%.15g\t%.15g\t%.15g\t%.15g\t%.15g\t%.15g"
                           "\t%d\t%d\t%d\t%d\t%d\t%.15g\n",
                           r.vortex, p[0], p[1], p[2], u[0], u[1], u[2], t[0], t[1], t[2], m[0], m[1], m[2], i,
                           v.links[2 * i + 1], v.links[2 * i], v.status[2 * i], v.status[2 * i + 1], v.dxi[i]);
  out.append(buf, len > 0 ? (size_t)len : 0);
}

bool write_text(const FrameView& v, const char* filename, std::string& err) {
  if (v.n > 0 && (!v.vels || !v.tan || !v.nrm || !v.dxi)) {
    err = "text frames need vels, tangents, normals and dxi";
    return false;
  }
  std::vector<Row> rows;
  if (!frame_order(v, rows)) {
    err = "the tangle's links do not close into vortices";
    return false;
  }
  const size_t nr = rows.size();
  unsigned nt = std::max(1u, std::thread::hardware_concurrency());
  nt = (unsigned)std::min<size_t>(nt, std::max<size_t>(1, nr / 4096));
  std::vector<std::string> parts(nt);
  std::vector<std::thread> pool;
  for (unsigned w = 0; w < nt; ++w)
    pool.emplace_back([&, w] {
      const size_t lo = nr * w / nt, hi = nr * (w + 1) / nt;
      parts[w].reserve((hi - lo) * 330);
      for (size_t r = lo; r < hi; ++r) format_row(v, rows[r], parts[w]);
    });
  for (auto& th : pool) th.join();
  FILE* f = fopen(filename, "w");
  if (!f) {
    err = std::string("cannot open ") + filename;
    return false;
  }
  bool ok = true;
  for (const auto& s : parts) ok = ok && fwrite(s.data(), 1, s.size(), f) == s.size();
  ok = (fclose(f) == 0) && ok;
  if (!ok) err = std::string("write failed: ") + filename;
  return ok;
}

bool write_binary(const FrameView& v, const ov_frame_header& h, const char* filename, std::string& err) {
  FILE* f = fopen(filename, "wb");
  if (!f) {
    err = std::string("cannot open ") + filename;
    return false;
  }
  const size_t n = (size_t)v.n;
  const double zeros[64] = {0};
  auto put = [&](const void* p, size_t bytes) {
    if (p) return fwrite(p, 1, bytes, f) == bytes;
    // an array the tangle does not have: zeros
    for (size_t done = 0; done < bytes;) {
      const size_t b = std::min(bytes - done, sizeof(zeros));
      if (fwrite(zeros, 1, b, f) != b) return false;
      done += b;
    }
    return true;
  };
  bool ok = put(&h, sizeof(h)) && put(v.pos, 24 * n) && put(v.vels, 24 * n) && put(v.tan, 24 * n) &&
            put(v.nrm, 24 * n) && put(v.dxi, 8 * n) && put(v.links, 8 * n) && put(v.status, 8 * n);
  ok = (fclose(f) == 0) && ok;
  if (!ok) err = std::string("write failed: ") + filename;
  return ok;
}

ov_frame_header header_of(int n, double time, const double lo[3], const double hi[3], const int wall[6]) {
  ov_frame_header h;
  memset(&h, 0, sizeof(h));
  memcpy(h.magic, "OVFRAME", 8);
  h.version = 1;
  h.n = n;
  h.time = time;
  for (int c = 0; c < 3; ++c) {
    h.box_lo[c] = lo[c];
    h.box_hi[c] = hi[c];
  }
  for (int f = 0; f < 6; ++f) h.wall[f] = wall[f];
  return h;
}

bool read_header(FILE* f, ov_frame_header& h) {
  if (fread(&h, 1, sizeof(h), f) != sizeof(h)) return false;
  return memcmp(h.magic, "OVFRAME", 8) == 0 && h.version == 1 && h.n >= 0;
}

// ---------------------------------------------------------------- writers
// A frame of a device-resident state on its way to a file.
struct FrameJob {
  int device = 0;
  cudaEvent_t copied = nullptr;   // the pinned copy is complete
  std::thread writer;
  std::string err;
  bool ok = true;
};

struct FrameSlot {
  DevBuf snap;                    // device snapshot of the slot arrays
  char* host = nullptr;           // pinned copy
  size_t host_bytes = 0;
  cudaStream_t copy = nullptr;
  cudaEvent_t taken = nullptr, copied = nullptr;
  std::unique_ptr<FrameJob> job;
  ~FrameSlot() {
    wait();
    if (host) cudaFreeHost(host);
    if (copy) cudaStreamDestroy(copy);
    if (taken) cudaEventDestroy(taken);
    if (copied) cudaEventDestroy(copied);
  }
  bool wait() {
    if (!job) return true;
    if (job->writer.joinable()) job->writer.join();
    const bool ok = job->ok;
    if (!ok) ov_set_error(OV_ERR_INVALID, "frame write: %s", job->err.c_str());
    job.reset();
    return ok;
  }
};

std::mutex g_slots_mu;
std::vector<FrameSlot*> g_slots;   // every slot with a write that may be pending

}  // namespace

// Frame buffers of a state (created on first use, released with the state).
void ov_frames_release(ov_state_impl* s) {
  if (!s->frames) return;
  FrameSlot* fs = static_cast<FrameSlot*>(s->frames);
  {
    std::lock_guard<std::mutex> lk(g_slots_mu);
    for (auto& p : g_slots)
      if (p == fs) p = nullptr;
  }
  delete fs;
  s->frames = nullptr;
}

extern "C" {

int ov_save_frame(const struct tangle_state* tangle, const char* filename, double time, int format) {
  ov_clear_error();
  if (!tangle || !filename || tangle->N < 0 ||
      (tangle->N > 0 && (!tangle->vnodes || !tangle->connections || !tangle->status))) {
    ov_set_error(OV_ERR_INVALID, "ov_save_frame: null tangle, arrays or file name");
    return -OV_ERR_INVALID;
  }
  const FrameView v = view_of(tangle);
  std::string err;
  bool ok;
  if (format == OV_FRAME_TEXT) {
    ok = write_text(v, filename, err);
  } else if (format == OV_FRAME_BINARY) {
    double lo[3], hi[3];
    int wall[6];
    for (int c = 0; c < 3; ++c) {
      lo[c] = tangle->box.bottom_left_back.p[c];
      hi[c] = tangle->box.top_right_front.p[c];
    }
    for (int f = 0; f < 6; ++f) wall[f] = tangle->box.wall[f];
    ok = write_binary(v, header_of(tangle->N, time, lo, hi, wall), filename, err);
  } else {
    ov_set_error(OV_ERR_INVALID, "ov_save_frame: unknown format %d", format);
    return -OV_ERR_INVALID;
  }
  if (!ok) {
    ov_set_error(OV_ERR_INVALID, "ov_save_frame: %s", err.c_str());
    return -OV_ERR_INVALID;
  }
  return 0;
}

int ov_save_tangle(const struct tangle_state* tangle, const char* filename) {
  return ov_save_frame(tangle, filename, 0.0, OV_FRAME_TEXT);
}

int ov_state_save_frame(ov_state* st, const char* filename, double time, int format) {
  ov_clear_error();
  if (!st || !filename || (format != OV_FRAME_TEXT && format != OV_FRAME_BINARY)) {
    ov_set_error(OV_ERR_INVALID, "ov_state_save_frame: null state or file name, or unknown format");
    return -OV_ERR_INVALID;
  }
  ov_state_impl* s = ov_state_impl_of(st);
  if (!s->frames) {
    s->frames = new FrameSlot();
    std::lock_guard<std::mutex> lk(g_slots_mu);
    g_slots.push_back(static_cast<FrameSlot*>(s->frames));
  }
  FrameSlot* fs = static_cast<FrameSlot*>(s->frames);
  if (!fs->wait()) return -ov_last_error();   // the previous frame of this state
  if (!fs->copy) {
    OV_TRY_CUDA(cudaStreamCreateWithFlags(&fs->copy, cudaStreamNonBlocking));
    OV_TRY_CUDA(cudaEventCreateWithFlags(&fs->taken, cudaEventDisableTiming));
    OV_TRY_CUDA(cudaEventCreateWithFlags(&fs->copied, cudaEventDisableTiming));
  }
  const size_t n = (size_t)s->n;
  // layout of the snapshot (device and pinned): pos, vels, tan, nrm, dxi, links, status
  const size_t off[8] = {0, 24 * n, 48 * n, 72 * n, 96 * n, 104 * n, 112 * n, 120 * n};
  const size_t bytes = std::max<size_t>(off[7], 16);
  if (!fs->snap.reserve(bytes)) return -ov_last_error();
  if (bytes > fs->host_bytes) {
    if (fs->host) cudaFreeHost(fs->host);
    fs->host = nullptr;
    fs->host_bytes = 0;
    OV_TRY_CUDA(cudaMallocHost(&fs->host, bytes));
    fs->host_bytes = bytes;
  }
  char* d = static_cast<char*>(fs->snap.p);
  const DevBuf* src[7] = {&s->pos, &s->vels, &s->tan, &s->nrm, &s->dxi, &s->links, &s->status};
  if (n) {
    for (int a = 0; a < 7; ++a)
      OV_TRY_CUDA(cudaMemcpyAsync(d + off[a], src[a]->p, off[a + 1] - off[a], cudaMemcpyDeviceToDevice, s->stream));
  }
  OV_TRY_CUDA(cudaEventRecord(fs->taken, s->stream));
  OV_TRY_CUDA(cudaStreamWaitEvent(fs->copy, fs->taken, 0));
  if (n) OV_TRY_CUDA(cudaMemcpyAsync(fs->host, d, off[7], cudaMemcpyDeviceToHost, fs->copy));
  OV_TRY_CUDA(cudaEventRecord(fs->copied, fs->copy));

  auto job = std::make_unique<FrameJob>();
  OV_TRY_CUDA(cudaGetDevice(&job->device));
  job->copied = fs->copied;
  FrameView v;
  v.n = (int)n;
  const char* h = fs->host;
  v.pos = reinterpret_cast<const double*>(h + off[0]);
  v.vels = reinterpret_cast<const double*>(h + off[1]);
  v.tan = reinterpret_cast<const double*>(h + off[2]);
  v.nrm = reinterpret_cast<const double*>(h + off[3]);
  v.dxi = reinterpret_cast<const double*>(h + off[4]);
  v.links = reinterpret_cast<const int*>(h + off[5]);
  v.status = reinterpret_cast<const int*>(h + off[6]);
  int wall[6];
  for (int f = 0; f < 6; ++f) wall[f] = s->walls[f];
  const ov_frame_header hd = header_of((int)n, time, s->P.lo, s->P.hi, wall);
  const std::string name(filename);
  FrameJob* jp = job.get();
  jp->writer = std::thread([jp, v, hd, name, format] {
    cudaSetDevice(jp->device);
    if (cudaEventSynchronize(jp->copied) != cudaSuccess) {
      jp->ok = false;
      jp->err = "device copy of the frame failed";
      return;
    }
    jp->ok = format == OV_FRAME_TEXT ? write_text(v, name.c_str(), jp->err)
                                     : write_binary(v, hd, name.c_str(), jp->err);
  });
  fs->job = std::move(job);
  return 0;
}

int ov_frame_wait(void) {
  ov_clear_error();
  std::vector<FrameSlot*> slots;
  {
    std::lock_guard<std::mutex> lk(g_slots_mu);
    slots = g_slots;
  }
  bool ok = true;
  for (FrameSlot* fs : slots)
    if (fs) ok = fs->wait() && ok;
  return ok ? 0 : -ov_last_error();
}

int ov_frame_info(const char* filename, int* n, double* time) {
  ov_clear_error();
  FILE* f = filename ? fopen(filename, "rb") : nullptr;
  if (!f) {
    ov_set_error(OV_ERR_INVALID, "ov_frame_info: cannot open %s", filename ? filename : "(null)");
    return -OV_ERR_INVALID;
  }
  ov_frame_header h;
  const bool ok = read_header(f, h);
  fclose(f);
  if (!ok) {
    ov_set_error(OV_ERR_INVALID, "ov_frame_info: %s is not a binary frame", filename);
    return -OV_ERR_INVALID;
  }
  if (n) *n = h.n;
  if (time) *time = h.time;
  return 0;
}

int ov_load_frame(const char* filename, struct tangle_state* tangle, double* time) {
  ov_clear_error();
  FILE* f = filename && tangle ? fopen(filename, "rb") : nullptr;
  if (!f) {
    ov_set_error(OV_ERR_INVALID, "ov_load_frame: null tangle or cannot open the file");
    return -OV_ERR_INVALID;
  }
  ov_frame_header h;
  bool ok = read_header(f, h);
  if (ok && h.n != tangle->N) {
    fclose(f);
    ov_set_error(OV_ERR_INVALID, "ov_load_frame: the frame has %d slots, the tangle %d", h.n, tangle->N);
    return -OV_ERR_INVALID;
  }
  const size_t n = (size_t)h.n;
  auto get = [&](void* p, size_t bytes) {
    if (p) return fread(p, 1, bytes, f) == bytes;
    return fseek(f, (long)bytes, SEEK_CUR) == 0;   // an array the tangle does not have
  };
  ok = ok && get(tangle->vnodes, 24 * n) && get(tangle->vels, 24 * n) && get(tangle->tangents, 24 * n) &&
       get(tangle->normals, 24 * n) && get(tangle->dxi, 8 * n) && get(tangle->connections, 8 * n) &&
       get(tangle->status, 8 * n);
  fclose(f);
  if (!ok) {
    ov_set_error(OV_ERR_INVALID, "ov_load_frame: %s is not a complete binary frame", filename);
    return -OV_ERR_INVALID;
  }
  for (int c = 0; c < 3; ++c) {
    tangle->box.bottom_left_back.p[c] = h.box_lo[c];
    tangle->box.top_right_front.p[c] = h.box_hi[c];
  }
  for (int w = 0; w < 6; ++w) tangle->box.wall[w] = (wall_type)h.wall[w];
  if (time) *time = h.time;
  return 0;
}

}  // extern "C"
