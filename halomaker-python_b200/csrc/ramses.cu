// RAMSES particle files -> the dense particle arrays the finder reads, with
// the decode on the device.
//
// Replaces _read_ramses_new_1010 (src/input_output.py:624-760) and the two
// passes read_ramses_new_101 drives it through (input_output.py:856-989),
// stellar payload off:
//   * records per part file (Fortran sequential, 4-byte lengths around each):
//     ncpu, ndim, npart, localseed, nstar, mstar_tot, mstar_lost, nsink,
//     x, y, z, vx, vy, vz, mass, id (int32), level, Ra4: family (int8), tag;
//     then, when nstar > 0 or nsink > 0, Ra3 files hold the birth time, which
//     classifies families there;
//   * families: Ra4 dm = family 1, star = family 2; Ra3 dm = id > 0 and birth
//     time 0, star = (birth < 0 and id > 0) or (birth != 0 and id < 0);
//   * dense layout: ind = |id| (+ ndm for stars when family = all) - 1;
//     pos = x - 0.5, vel = v * scale_l / scale_t * 1e-5, mass = m, and
//     source_pid = |id| for a single family;
//   * errors as the reference raises them: a file whose selected ind leave
//     [0, nselected) or repeat inside the file; for a single family, slots
//     left unwritten (cross-file repeats); no particle selected.
// The host walks each file's record lengths (validating head == tail, as
// skip_records does), reads the file once into pinned memory and copies the
// payloads it needs to the device (double-buffered against the next file's
// read); the reference reads every file twice (count pass, load pass).  The
// family counts come from one device pass over all files, the scatter from
// one launch per file in file order, so a later file overwrites an earlier
// one exactly where the reference's loop would.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "engine.h"

namespace ahop {
namespace {

enum { R_X = 0, R_Y, R_Z, R_VX, R_VY, R_VZ, R_M, R_ID, R_FAM, R_TB, R_N };

struct PartFile {
  int64_t npart = 0;
  int64_t first = 0;        // index of its first particle over all files
  int64_t dev[R_N] = {};    // device byte offset of each payload in the staging area, -1 if absent
  int64_t file_off[R_N] = {};
  int64_t bytes = 0;        // file size
};

struct DevFile {  // per-file view for the kernels
  const double *x, *y, *z, *vx, *vy, *vz, *m, *tb;
  const int32_t* id;
  const int8_t* fam;
  int64_t npart, first;
};

struct RamsesState {
  bool open = false;
  AhopRamsesParams prm{};
  AhopRamsesCounts counts{};
  std::vector<PartFile> files;
  std::vector<std::string> paths;
  DevBuf d_raw, d_files, d_cnt, d_owner, d_flag;
  HostBuf h_stage[2];
  cudaEvent_t ev[2] = {};
  cudaStream_t st = nullptr;
};

RamsesState& rstate() {
  static RamsesState* s = new RamsesState();
  return *s;
}

__device__ __forceinline__ void classify(const DevFile& F, int version, int64_t k, bool& dm, bool& star) {
  const int32_t id = F.id[k];
  if (version == 4) {
    const int8_t f = F.fam[k];
    dm = f == 1;
    star = f == 2;
  } else {
    const double t = F.tb ? F.tb[k] : 0.0;
    dm = id > 0 && t == 0.0;
    star = (t < 0.0 && id > 0) || (t != 0.0 && id < 0);
  }
}

// Family counts per file: cnt[2 f] = dark matter, cnt[2 f + 1] = stars.
__global__ void count_kernel(const DevFile* __restrict__ files, int nfiles, int version, int64_t total,
                             unsigned long long* __restrict__ cnt) {
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int f = -1;
  bool dm = false, star = false;
  if (g < total) {
    int lo = 0, hi = nfiles - 1;  // last file whose first <= g
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (files[mid].first <= g) lo = mid; else hi = mid - 1;
    }
    f = lo;
    classify(files[f], version, g - files[f].first, dm, star);
  }
  // files are contiguous in g, so most warps see one file: aggregate per file
  // value among the lanes that share it
  const unsigned act = __ballot_sync(0xffffffffu, f >= 0);
  if (f >= 0) {
    const unsigned same = __match_any_sync(act, f);
    const unsigned ndm = __popc(__ballot_sync(act, dm) & same);
    const unsigned nst = __popc(__ballot_sync(act, star) & same);
    if ((threadIdx.x & 31) == __ffs(same) - 1) {
      if (ndm) atomicAdd(&cnt[2 * f], (unsigned long long)ndm);
      if (nst) atomicAdd(&cnt[2 * f + 1], (unsigned long long)nst);
    }
  }
}

// Scatter of one file.  flag[0]: first file with a bad index + 1; flag[1]:
// a repeated index inside one file (file + 1).
__global__ void scatter_kernel(DevFile F, int fidx, int version, int family, int64_t ndm_all, int64_t nsel,
                               double scale_l, double scale_t, double* __restrict__ pos, double* __restrict__ vel,
                               double* __restrict__ mass, int64_t* __restrict__ spid, int32_t* __restrict__ owner,
                               int32_t* __restrict__ flag) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= F.npart) return;
  bool dm, star;
  classify(F, version, k, dm, star);
  const bool sel = family == 0 ? (dm || star) : (family == 1 ? dm : star);
  if (!sel) return;
  const int32_t id = F.id[k];
  const int64_t src = id < 0 ? -(int64_t)id : (int64_t)id;
  const int64_t loc = (family == 0 && star) ? src + ndm_all : src;
  const int64_t ind = loc - 1;
  if (ind < 0 || ind >= nsel) {
    atomicCAS(&flag[0], 0, fidx + 1);
    return;
  }
  if (atomicExch(&owner[ind], fidx) == fidx) atomicCAS(&flag[1], 0, fidx + 1);
  pos[3 * ind] = __dsub_rn(F.x[k], 0.5);
  pos[3 * ind + 1] = __dsub_rn(F.y[k], 0.5);
  pos[3 * ind + 2] = __dsub_rn(F.z[k], 0.5);
  // v * scale_l / scale_t * 1e-5, left to right
  vel[3 * ind] = __dmul_rn(__ddiv_rn(__dmul_rn(F.vx[k], scale_l), scale_t), 1e-5);
  vel[3 * ind + 1] = __dmul_rn(__ddiv_rn(__dmul_rn(F.vy[k], scale_l), scale_t), 1e-5);
  vel[3 * ind + 2] = __dmul_rn(__ddiv_rn(__dmul_rn(F.vz[k], scale_l), scale_t), 1e-5);
  mass[ind] = F.m[k];
  if (spid) spid[ind] = src;
}

__global__ void unwritten_kernel(const int32_t* __restrict__ owner, int64_t n, unsigned long long* __restrict__ cnt) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool hole = i < n && owner[i] < 0;
  const unsigned b = __ballot_sync(0xffffffffu, hole);
  if ((threadIdx.x & 31) == 0 && b) atomicAdd(cnt, (unsigned long long)__popc(b));
}

// Record walker over one file: offsets of each record's payload.
struct Walker {
  FILE* f = nullptr;
  int64_t pos = 0, size = 0;
  std::string path, err;
  bool next(int64_t* off, int64_t* len) {
    if (pos + 4 > size) { err = "truncated record header"; return false; }
    uint32_t head = 0, tail = 0;
    if (fseek(f, (long)pos, SEEK_SET) || fread(&head, 4, 1, f) != 1) { err = "read failed"; return false; }
    if (pos + 8 + (int64_t)head > size) { err = "record runs past the end of the file"; return false; }
    if (fseek(f, (long)(pos + 4 + head), SEEK_SET) || fread(&tail, 4, 1, f) != 1) { err = "read failed"; return false; }
    if (head != tail) {
      err = "Sizes do not agree in the header(" + std::to_string(head) + ") and footer(" + std::to_string(tail) +
            ") for this record";
      return false;
    }
    *off = pos + 4;
    *len = head;
    pos += 8 + (int64_t)head;
    return true;
  }
  bool read_i32(int32_t* v) {
    int64_t o, n;
    if (!next(&o, &n)) return false;
    if (n < 4) { err = "integer record too short"; return false; }
    if (fseek(f, (long)o, SEEK_SET) || fread(v, 4, 1, f) != 1) { err = "read failed"; return false; }
    return true;
  }
  bool skip() {
    int64_t o, n;
    return next(&o, &n);
  }
};

int walk_file(const std::string& path, int version, PartFile& P) {
  Walker W;
  W.path = path;
  W.f = fopen(path.c_str(), "rb");
  if (!W.f) { set_error("cannot open " + path); return AHOP_EIO; }
  fseek(W.f, 0, SEEK_END);
  W.size = ftell(W.f);
  P.bytes = W.size;
  int32_t ncpu = 0, ndim = 0, npart = 0, nstar = 0, nsink = 0;
  bool ok = W.read_i32(&ncpu) && W.read_i32(&ndim) && W.read_i32(&npart) && W.skip() && W.read_i32(&nstar) &&
            W.skip() && W.skip() && W.read_i32(&nsink);
  auto fail = [&](const std::string& why) {
    fclose(W.f);
    set_error(path + ": " + why);
    return AHOP_EDATA;
  };
  if (!ok) return fail(W.err);
  if (ndim != 3) return fail("ndim " + std::to_string(ndim) + " (only 3 is supported)");
  if (npart < 0) return fail("negative npart");
  P.npart = npart;
  for (auto& v : P.file_off) v = -1;
  auto take = [&](int r, int64_t elem) {
    int64_t o, n;
    if (!W.next(&o, &n)) return false;
    if (n != elem * (int64_t)npart) {
      W.err = "record of " + std::to_string(n) + " bytes, expected " + std::to_string(elem * (int64_t)npart);
      return false;
    }
    if (r >= 0) P.file_off[r] = o;
    return true;
  };
  ok = take(R_X, 8) && take(R_Y, 8) && take(R_Z, 8) && take(R_VX, 8) && take(R_VY, 8) && take(R_VZ, 8) &&
       take(R_M, 8) && take(R_ID, 4) && W.skip();
  if (ok && version == 4) ok = take(R_FAM, 1) && W.skip();
  if (ok && version != 4 && (nstar > 0 || nsink > 0)) ok = take(R_TB, 8);
  if (!ok) return fail(W.err);
  fclose(W.f);
  return AHOP_OK;
}

int64_t elem_bytes(int r) { return r == R_ID ? 4 : r == R_FAM ? 1 : 8; }

}  // namespace
}  // namespace ahop

using namespace ahop;

extern "C" int ahop_ramses_open(const char* const* paths, int32_t nfiles, const AhopRamsesParams* p,
                                AhopRamsesCounts* out) {
  RamsesState& S = rstate();
  S.open = false;
  if (!paths || nfiles <= 0 || !p || !out) { set_error("ramses_open: bad arguments"); return AHOP_EINVAL; }
  if (p->version != 3 && p->version != 4) { set_error("ramses version must be 3 or 4"); return AHOP_EINVAL; }
  if (p->family < 0 || p->family > 2) { set_error("family must be 0 (all), 1 (dm) or 2 (star)"); return AHOP_EINVAL; }
  if (!(p->scale_t != 0.0)) { set_error("scale_t must be non-zero"); return AHOP_EINVAL; }
  int dev = 0;
  AHOP_CUDA_TRY(cudaGetDevice(&dev));
  if (!S.st) {
    AHOP_CUDA_TRY(cudaStreamCreateWithFlags(&S.st, cudaStreamNonBlocking));
    for (auto& e : S.ev) AHOP_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  S.prm = *p;
  S.files.assign(nfiles, PartFile());
  S.paths.assign(paths, paths + nfiles);
  int rc;
  int64_t total = 0, dev_bytes = 0, max_file = 0;
  for (int f = 0; f < nfiles; ++f) {
    if ((rc = walk_file(S.paths[f], p->version, S.files[f]))) return rc;
    PartFile& P = S.files[f];
    P.first = total;
    total += P.npart;
    max_file = std::max(max_file, P.bytes);
    for (int r = 0; r < R_N; ++r) {
      P.dev[r] = -1;
      if (P.file_off[r] < 0) continue;
      P.dev[r] = dev_bytes;
      dev_bytes += ((elem_bytes(r) * P.npart + 255) / 256) * 256;
    }
  }
  AHOP_CUDA_TRY(S.d_raw.ensure((size_t)dev_bytes + 256));
  // read each file once into pinned memory (two buffers: the next read
  // overlaps the previous file's copies) and send the payloads
  for (int b = 0; b < 2; ++b) AHOP_CUDA_TRY(S.h_stage[b].ensure((size_t)max_file + 16));
  for (int f = 0; f < nfiles; ++f) {
    const int b = f & 1;
    if (f >= 2) AHOP_CUDA_TRY(cudaEventSynchronize(S.ev[b]));
    PartFile& P = S.files[f];
    FILE* fp = fopen(S.paths[f].c_str(), "rb");
    if (!fp) { set_error("cannot open " + S.paths[f]); return AHOP_EIO; }
    const size_t got = fread(S.h_stage[b].p, 1, (size_t)P.bytes, fp);
    fclose(fp);
    if ((int64_t)got != P.bytes) { set_error("short read of " + S.paths[f]); return AHOP_EIO; }
    for (int r = 0; r < R_N; ++r) {
      if (P.dev[r] < 0 || P.npart == 0) continue;
      AHOP_CUDA_TRY(cudaMemcpyAsync(S.d_raw.as<char>() + P.dev[r], S.h_stage[b].as<char>() + P.file_off[r],
                                    (size_t)(elem_bytes(r) * P.npart), cudaMemcpyHostToDevice, S.st));
    }
    AHOP_CUDA_TRY(cudaEventRecord(S.ev[b], S.st));
  }
  // per-file device views
  std::vector<DevFile> df(nfiles);
  char* raw = S.d_raw.as<char>();
  for (int f = 0; f < nfiles; ++f) {
    const PartFile& P = S.files[f];
    auto at = [&](int r) -> const void* { return P.dev[r] >= 0 ? raw + P.dev[r] : nullptr; };
    df[f] = DevFile{(const double*)at(R_X), (const double*)at(R_Y), (const double*)at(R_Z), (const double*)at(R_VX),
                    (const double*)at(R_VY), (const double*)at(R_VZ), (const double*)at(R_M), (const double*)at(R_TB),
                    (const int32_t*)at(R_ID), (const int8_t*)at(R_FAM), P.npart, P.first};
  }
  AHOP_CUDA_TRY(S.d_files.ensure(sizeof(DevFile) * nfiles));
  AHOP_CUDA_TRY(cudaMemcpyAsync(S.d_files.p, df.data(), sizeof(DevFile) * nfiles, cudaMemcpyHostToDevice, S.st));
  AHOP_CUDA_TRY(S.d_cnt.ensure(sizeof(unsigned long long) * (2 * (size_t)nfiles + 2)));
  AHOP_CUDA_TRY(cudaMemsetAsync(S.d_cnt.p, 0, sizeof(unsigned long long) * (2 * (size_t)nfiles + 2), S.st));
  if (total > 0) {
    count_kernel<<<(unsigned)((total + 255) / 256), 256, 0, S.st>>>(S.d_files.as<DevFile>(), nfiles, p->version,
                                                                    total, S.d_cnt.as<unsigned long long>());
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  std::vector<unsigned long long> cnt(2 * (size_t)nfiles);
  AHOP_CUDA_TRY(cudaMemcpyAsync(cnt.data(), S.d_cnt.p, cnt.size() * 8, cudaMemcpyDeviceToHost, S.st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(S.st));
  int64_t ndm = 0, nstar = 0;
  for (int f = 0; f < nfiles; ++f) {
    ndm += (int64_t)cnt[2 * f];
    nstar += (int64_t)cnt[2 * f + 1];
  }
  const int64_t nsel = p->family == 0 ? ndm + nstar : (p->family == 1 ? ndm : nstar);
  if (nsel == 0) { set_error("No particles selected for this family"); return AHOP_EDATA; }
  S.counts = AhopRamsesCounts{total, ndm, nstar, nsel, nfiles, 3};
  *out = S.counts;
  S.open = true;
  return AHOP_OK;
}

extern "C" int ahop_ramses_decode_device(double* d_pos, double* d_vel, double* d_mass, int64_t* d_source_pid,
                                         void* stream) {
  RamsesState& S = rstate();
  if (!S.open) { set_error("ramses_decode: no files open (call ahop_ramses_open first)"); return AHOP_ESTATE; }
  if (!d_pos || !d_vel || !d_mass) { set_error("ramses_decode: null output"); return AHOP_EINVAL; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t nsel = S.counts.nselected;
  const int fam = S.prm.family;
  // the staged payloads and counts were written on the reader's stream
  AHOP_CUDA_TRY(cudaStreamSynchronize(S.st));
  AHOP_CUDA_TRY(S.d_owner.ensure((size_t)nsel * 4 + 4));
  AHOP_CUDA_TRY(S.d_flag.ensure(64));
  AHOP_CUDA_TRY(cudaMemsetAsync(S.d_owner.p, 0xff, (size_t)nsel * 4, st));  // -1: not written
  AHOP_CUDA_TRY(cudaMemsetAsync(S.d_flag.p, 0, 64, st));
  // zero-filled outputs, as the reference's freshly allocated shared arrays
  AHOP_CUDA_TRY(cudaMemsetAsync(d_pos, 0, (size_t)nsel * 24, st));
  AHOP_CUDA_TRY(cudaMemsetAsync(d_vel, 0, (size_t)nsel * 24, st));
  AHOP_CUDA_TRY(cudaMemsetAsync(d_mass, 0, (size_t)nsel * 8, st));
  if (d_source_pid) AHOP_CUDA_TRY(cudaMemsetAsync(d_source_pid, 0xff, (size_t)nsel * 8, st));
  const int64_t ndm_all = fam == 0 ? S.counts.ndm : 0;
  char* raw = S.d_raw.as<char>();
  for (int f = 0; f < (int)S.files.size(); ++f) {
    const PartFile& P = S.files[f];
    if (P.npart == 0) continue;
    auto at = [&](int r) -> const void* { return P.dev[r] >= 0 ? raw + P.dev[r] : nullptr; };
    const DevFile F{(const double*)at(R_X), (const double*)at(R_Y), (const double*)at(R_Z), (const double*)at(R_VX),
                    (const double*)at(R_VY), (const double*)at(R_VZ), (const double*)at(R_M), (const double*)at(R_TB),
                    (const int32_t*)at(R_ID), (const int8_t*)at(R_FAM), P.npart, P.first};
    scatter_kernel<<<(unsigned)((P.npart + 255) / 256), 256, 0, st>>>(
        F, f, S.prm.version, fam, ndm_all, nsel, S.prm.scale_l, S.prm.scale_t, d_pos, d_vel, d_mass,
        fam == 0 ? nullptr : d_source_pid, S.d_owner.as<int32_t>(), S.d_flag.as<int32_t>());
    AHOP_CUDA_TRY(cudaGetLastError());
  }
  unsigned long long* holes = reinterpret_cast<unsigned long long*>(S.d_flag.as<char>() + 32);
  unwritten_kernel<<<(unsigned)((nsel + 255) / 256), 256, 0, st>>>(S.d_owner.as<int32_t>(), nsel, holes);
  AHOP_CUDA_TRY(cudaGetLastError());
  int32_t flag[2] = {0, 0};
  unsigned long long nholes = 0;
  AHOP_CUDA_TRY(cudaMemcpyAsync(flag, S.d_flag.p, 8, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaMemcpyAsync(&nholes, holes, 8, cudaMemcpyDeviceToHost, st));
  AHOP_CUDA_TRY(cudaStreamSynchronize(st));
  static const char* fname[3] = {"all", "dm", "star"};
  const int bad = flag[0] && flag[1] ? std::min(flag[0], flag[1]) : (flag[0] ? flag[0] : flag[1]);
  if (bad) {
    set_error(std::string("Non-dense or duplicate ") + fname[fam] + " particle IDs in icpu=" + std::to_string(bad));
    return AHOP_EDATA;
  }
  if (fam != 0 && nholes) {
    set_error(std::string("Incomplete or duplicate source PIDs for family=") + fname[fam]);
    return AHOP_EDATA;
  }
  return AHOP_OK;
}

extern "C" int ahop_ramses_close(void) {
  RamsesState& S = rstate();
  S.open = false;
  S.files.clear();
  S.paths.clear();
  S.d_raw.release();
  S.d_files.release();
  S.d_cnt.release();
  S.d_owner.release();
  S.d_flag.release();
  for (auto& h : S.h_stage) h.release();
  return AHOP_OK;
}
