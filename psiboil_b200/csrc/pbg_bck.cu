// Checkpoint files in the reference's .bck format: reading reference states
// as inputs and writing the engine's results where the reference can load
// them.
//
// Format (Scalar::save / Scalar::load, Src/Field/Scalar/scalar_save.cpp:20-32,
// scalar_load.cpp:26-37): per field, three ints (the block's extents ni, nj,
// nk, the BW = 3 halo included) and then the block's ni*nj*nk doubles in
// val[0][0] order (k fastest). A Centered checkpoint is phi followed by cold
// (centered_save.cpp:4-23). File names follow name_file
// (Src/Global/global_name_file.cpp:4-33): base, "_p" and the processor number
// in 3 digits, "_" and the step in 6 digits, ".bck" (each part only when its
// number is > -1).
//
// The reference's load ignores the stored extents; reading here checks them
// against the expected block and fails on a mismatch or a short file.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/psiboil_b200.h"

namespace pbg {
void set_last_error(const char *msg);  // pbg_capi.cu
}

namespace {

constexpr int kBW = 3;  // the reference's halo width (global_buffer_width.cpp:4)

int bfail(int code, const std::string &m) {
  pbg::set_last_error(m.c_str());
  return code;
}

bool copy_in(double *dst, const double *src, size_t n, int where) {
  if (where == PBG_DEVICE) return cudaMemcpy(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost) == cudaSuccess;
  std::memcpy(dst, src, n * sizeof(double));
  return true;
}

bool copy_out(double *dst, const double *src, size_t n, int where) {
  if (where == PBG_DEVICE) return cudaMemcpy(dst, src, n * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess;
  std::memcpy(dst, src, n * sizeof(double));
  return true;
}

int write_blocks(const char *path, int nfields, const std::vector<const double *> &blocks, int ni, int nj, int nk) {
  std::ofstream out(path, std::ios::binary);
  if (!out) return bfail(PBG_ERR_ARG, std::string("bck: cannot open ") + path + " for writing");
  const size_t n = (size_t)ni * nj * nk;
  for (int f = 0; f < nfields; ++f) {
    out.write(reinterpret_cast<const char *>(&ni), sizeof(int));
    out.write(reinterpret_cast<const char *>(&nj), sizeof(int));
    out.write(reinterpret_cast<const char *>(&nk), sizeof(int));
    out.write(reinterpret_cast<const char *>(blocks[f]), n * sizeof(double));
  }
  if (!out) return bfail(PBG_ERR_STATE, std::string("bck: write failed: ") + path);
  return PBG_OK;
}

int read_blocks(const char *path, int nfields, std::vector<std::vector<double>> &blocks, int ni, int nj, int nk) {
  std::ifstream in(path, std::ios::binary);
  if (!in) return bfail(PBG_ERR_ARG, std::string("bck: cannot open ") + path);
  const size_t n = (size_t)ni * nj * nk;
  blocks.assign(nfields, std::vector<double>(n));
  for (int f = 0; f < nfields; ++f) {
    int e[3] = {0, 0, 0};
    in.read(reinterpret_cast<char *>(e), sizeof(e));
    if (!in) return bfail(PBG_ERR_ARG, std::string("bck: short file ") + path);
    if (e[0] != ni || e[1] != nj || e[2] != nk) {
      char m[256];
      std::snprintf(m, sizeof(m), "bck: field %d of %s is %d x %d x %d, expected %d x %d x %d", f, path, e[0],
                    e[1], e[2], ni, nj, nk);
      return bfail(PBG_ERR_ARG, m);
    }
    in.read(reinterpret_cast<char *>(blocks[f].data()), n * sizeof(double));
    if (!in) return bfail(PBG_ERR_ARG, std::string("bck: short file ") + path);
  }
  return PBG_OK;
}

// block extents of an interior grid (a unit extent is a dummy direction
// of a 2-D case, which the reference still pads with the halo)
void block_dims(int nx, int ny, int nz, int &ni, int &nj, int &nk) {
  ni = nx + 2 * kBW;
  nj = ny + 2 * kBW;
  nk = nz + 2 * kBW;
}

}  // namespace

extern "C" {

int pbg_bck_name(const char *base, int step, int cpu, char *out, int cap) {
  if (!base || !out || cap < 1) return bfail(PBG_ERR_ARG, "bck: bad arguments");
  std::ostringstream s;
  s << base;
  if (cpu > -1) {
    s << "_p";
    s.fill('0');
    s.width(3);
    s << cpu;
  }
  if (step > -1) {
    s << "_";
    s.fill('0');
    s.width(6);
    s << step;
  }
  s << ".bck";
  const std::string r = s.str();
  if ((int)r.size() + 1 > cap) return bfail(PBG_ERR_ARG, "bck: name buffer too small");
  std::memcpy(out, r.c_str(), r.size() + 1);
  return PBG_OK;
}

int pbg_bck_write(const char *path, int nfields, const double *const *fields, int ni, int nj, int nk, int where) {
  if (!path || !fields || nfields < 1 || ni < 1 || nj < 1 || nk < 1) return bfail(PBG_ERR_ARG, "bck: bad arguments");
  const size_t n = (size_t)ni * nj * nk;
  std::vector<std::vector<double>> host(nfields, std::vector<double>(n));
  std::vector<const double *> b(nfields);
  for (int f = 0; f < nfields; ++f) {
    if (!fields[f]) return bfail(PBG_ERR_ARG, "bck: NULL field");
    if (!copy_in(host[f].data(), fields[f], n, where)) return bfail(PBG_ERR_CUDA, "bck: device copy failed");
    b[f] = host[f].data();
  }
  return write_blocks(path, nfields, b, ni, nj, nk);
}

int pbg_bck_read(const char *path, int nfields, double *const *fields, int ni, int nj, int nk, int where) {
  if (!path || !fields || nfields < 1 || ni < 1 || nj < 1 || nk < 1) return bfail(PBG_ERR_ARG, "bck: bad arguments");
  std::vector<std::vector<double>> blocks;
  int rc = read_blocks(path, nfields, blocks, ni, nj, nk);
  if (rc != PBG_OK) return rc;
  for (int f = 0; f < nfields; ++f) {
    if (!fields[f]) return bfail(PBG_ERR_ARG, "bck: NULL field");
    if (!copy_out(fields[f], blocks[f].data(), blocks[f].size(), where)) return bfail(PBG_ERR_CUDA, "bck: device copy failed");
  }
  return PBG_OK;
}

int pbg_bck_write_compact(const char *path, int nfields, const double *const *fields, int nx, int ny, int nz,
                          int where) {
  if (!path || !fields || nfields < 1 || nx < 1 || ny < 1 || nz < 1) return bfail(PBG_ERR_ARG, "bck: bad arguments");
  int ni, nj, nk;
  block_dims(nx, ny, nz, ni, nj, nk);
  const size_t N = (size_t)nx * ny * nz, n = (size_t)ni * nj * nk;
  std::vector<std::vector<double>> blocks(nfields, std::vector<double>(n, 0.0));
  std::vector<double> c(N);
  std::vector<const double *> b(nfields);
  for (int f = 0; f < nfields; ++f) {
    if (!fields[f]) return bfail(PBG_ERR_ARG, "bck: NULL field");
    if (!copy_in(c.data(), fields[f], N, where)) return bfail(PBG_ERR_CUDA, "bck: device copy failed");
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j)
        std::memcpy(&blocks[f][(((size_t)(i + kBW) * nj) + j + kBW) * nk + kBW], &c[((size_t)i * ny + j) * nz],
                    nz * sizeof(double));
    b[f] = blocks[f].data();
  }
  return write_blocks(path, nfields, b, ni, nj, nk);
}

int pbg_bck_read_compact(const char *path, int nfields, double *const *fields, int nx, int ny, int nz, int where) {
  if (!path || !fields || nfields < 1 || nx < 1 || ny < 1 || nz < 1) return bfail(PBG_ERR_ARG, "bck: bad arguments");
  int ni, nj, nk;
  block_dims(nx, ny, nz, ni, nj, nk);
  std::vector<std::vector<double>> blocks;
  int rc = read_blocks(path, nfields, blocks, ni, nj, nk);
  if (rc != PBG_OK) return rc;
  const size_t N = (size_t)nx * ny * nz;
  std::vector<double> c(N);
  for (int f = 0; f < nfields; ++f) {
    if (!fields[f]) return bfail(PBG_ERR_ARG, "bck: NULL field");
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j)
        std::memcpy(&c[((size_t)i * ny + j) * nz], &blocks[f][(((size_t)(i + kBW) * nj) + j + kBW) * nk + kBW],
                    nz * sizeof(double));
    if (!copy_out(fields[f], c.data(), N, where)) return bfail(PBG_ERR_CUDA, "bck: device copy failed");
  }
  return PBG_OK;
}

}  // extern "C"
