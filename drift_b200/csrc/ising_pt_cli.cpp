// ising_pt_cli.cpp - command-line twin of the reference's GPU engine executable, on this library.
//
//   ising_pt <problem.bin> <result.bin>
//
// Reads the problem file that drift/gpu.py:86-95 writes (little-endian, packed:
// <Q seed, i n, i R, i n_rounds, i sweeps_per_round, i nnz, i k, f T_min, f T_max>, then
// int32 row_ptr[n+1], int32 col_idx[nnz], float weight[nnz], float h[n], int32 color_ptr[k+1],
// int32 color_spins[n]), runs the whole PT job through drift_pt_solve, and writes the result file
// drift/gpu.py:101-103 reads (double best_E, float best_s[n]). stderr gets the line whose
// `time=...s` and `throughput=...` fields drift/gpu.py:105-106 parses. Exit status 0 on success,
// 1 with a message on any error (the reference's convention, cuda/ising_pt.cu:30-38,133-136), so
// gpu_binary_path() can point at this program with no change to DRiFT.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/drift_pt.h"

namespace {

bool read_file(const char* path, std::vector<unsigned char>& out) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  unsigned char chunk[1 << 16];
  size_t got;
  while ((got = std::fread(chunk, 1, sizeof chunk, f)) > 0) out.insert(out.end(), chunk, chunk + got);
  const bool ok = !std::ferror(f);
  std::fclose(f);
  return ok;
}

template <typename T>
bool take(const std::vector<unsigned char>& buf, size_t& at, T& v) {
  if (at + sizeof(T) > buf.size()) return false;
  std::memcpy(&v, buf.data() + at, sizeof(T));
  at += sizeof(T);
  return true;
}

template <typename T>
bool take_array(const std::vector<unsigned char>& buf, size_t& at, size_t count, std::vector<T>& v) {
  if (count > (buf.size() - at) / sizeof(T)) return false;
  v.resize(count);
  if (count) std::memcpy(v.data(), buf.data() + at, count * sizeof(T));
  at += count * sizeof(T);
  return true;
}

int fail(const char* msg) {
  std::fprintf(stderr, "ising_pt: %s\n", msg);
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s <problem.bin> <result.bin>\n", argv[0]);
    return 1;
  }
  std::vector<unsigned char> buf;
  if (!read_file(argv[1], buf)) return fail("cannot read the problem file");
  size_t at = 0;
  uint64_t seed = 0;
  int32_t n = 0, R = 0, n_rounds = 0, spr = 0, nnz = 0, k = 0;
  float T_min = 0.0f, T_max = 0.0f;
  if (!take(buf, at, seed) || !take(buf, at, n) || !take(buf, at, R) || !take(buf, at, n_rounds) ||
      !take(buf, at, spr) || !take(buf, at, nnz) || !take(buf, at, k) || !take(buf, at, T_min) || !take(buf, at, T_max))
    return fail("problem file shorter than its 40-byte header");
  if (n < 1 || R < 1 || n_rounds < 0 || spr < 1 || nnz < 0 || k < 1 || k > n)
    return fail("problem header out of range (need n >= 1, R >= 1, n_rounds >= 0, sweeps >= 1, 1 <= k <= n)");
  std::vector<int32_t> row_ptr, col_idx, color_ptr, color_spins;
  std::vector<float> weight, h;
  if (!take_array(buf, at, (size_t)n + 1, row_ptr) || !take_array(buf, at, (size_t)nnz, col_idx) ||
      !take_array(buf, at, (size_t)nnz, weight) || !take_array(buf, at, (size_t)n, h) ||
      !take_array(buf, at, (size_t)k + 1, color_ptr) || !take_array(buf, at, (size_t)n, color_spins))
    return fail("problem file shorter than its header announces");
  if (at != buf.size()) return fail("problem file longer than its header announces");

  DriftPtCsr csr;
  csr.n = n;
  csr.nnz = nnz;
  csr.row_ptr = row_ptr.data();
  csr.col_idx = col_idx.data();
  csr.weight = weight.data();
  csr.h = h.data();
  csr.n_colors = k;
  csr.color_ptr = color_ptr.data();
  csr.color_spins = color_spins.data();
  DriftPtSolveArgs args;
  std::memset(&args, 0, sizeof args);
  args.n_replicas = R;
  args.n_rounds = n_rounds;
  args.sweeps_per_round = spr;
  args.seed = seed;
  args.T_min = T_min;
  args.T_max = T_max;
  std::vector<float> best_s((size_t)n);
  DriftPtSolveResult res;
  std::memset(&res, 0, sizeof res);
  res.best_s = best_s.data();
  if (drift_pt_solve(&csr, &args, &res) != DRIFT_PT_OK) {
    std::fprintf(stderr, "ising_pt: %s\n", drift_pt_last_error());
    return 1;
  }
  FILE* out = std::fopen(argv[2], "wb");
  if (!out) return fail("cannot write the result file");
  const bool ok = std::fwrite(&res.best_E, sizeof(double), 1, out) == 1 &&
                  std::fwrite(best_s.data(), sizeof(float), (size_t)n, out) == (size_t)n;
  if (std::fclose(out) != 0 || !ok) return fail("cannot write the result file");
  const double flips = (double)R * n_rounds * spr * n;
  std::fprintf(stderr,
               "best_E=%.6f  replicas=%d  n=%d  nnz=%d  colours=%d  flips=%.3e  time=%.6fs  throughput=%.6e flips/s  "
               "swap_rate=%.4f  engine=%s\n",
               res.best_E, R, n, nnz, k, flips, res.seconds, res.throughput, res.swap_rate, drift_pt_version());
  return 0;
}
