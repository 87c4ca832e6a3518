// uc_main — command-line driver with the reference's interface:
//
//   uc_main <k-mer file> k l <output file> [--config <file>] [--device N] [--sorted] [--check]
//
// (driver.cpp:422-432: exactly four positional arguments, no defaults).  The
// unitig lines are appended to the output file as the reference does
// (compact.h:10,25).  The reference ships three config files (base_config.txt,
// cond_config.txt, fourpart_config.txt) that none of its code reads; --config
// accepts a file of that form (six numeric lines, then one word), rejects
// anything else, and changes nothing.  Phase times are printed like the
// reference's timers (driver.cpp:641-657), ending with its "Total time:" line
// (driver.cpp:657: input read to output written).  --sorted writes the lines
// in byte order, so that equal input gives byte-equal output.  --check
// validates the arguments, the config file and the input's count line, and
// exits without touching a GPU.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "uc.h"

// The reference's config files: six lines that are each one number (integer
// or floating point, surrounding blanks allowed), then one line holding a
// single word, and nothing after it but blank lines.
static bool is_number(const std::string& s) {
  const char* b = s.c_str();
  char* end = nullptr;
  std::strtod(b, &end);
  if (end == b) return false;
  while (*end == ' ' || *end == '\t' || *end == '\r') ++end;
  return *end == '\0';
}

static bool is_word(const std::string& s) {
  size_t i = 0, n = s.size();
  while (i < n && (s[i] == ' ' || s[i] == '\t')) ++i;
  size_t j = n;
  while (j > i && (s[j - 1] == ' ' || s[j - 1] == '\t' || s[j - 1] == '\r')) --j;
  if (j == i) return false;
  for (size_t t = i; t < j; ++t)
    if (s[t] == ' ' || s[t] == '\t') return false;
  return true;
}

static bool check_config(const char* path) {
  std::ifstream f(path);
  if (!f.is_open()) return false;
  std::vector<std::string> lines;
  std::string s;
  while (std::getline(f, s)) lines.push_back(s);
  while (!lines.empty() && !is_word(lines.back()) &&
         lines.back().find_first_not_of(" \t\r") == std::string::npos)
    lines.pop_back();
  if (lines.size() != 7) return false;
  for (size_t i = 0; i < 6; ++i)
    if (!is_number(lines[i])) return false;
  return is_word(lines[6]);
}

// The input's count line (driver.cpp:296-304): digits, then the line's end.
static bool check_input(const char* path, unsigned long long* n) {
  std::ifstream f(path);
  if (!f.is_open()) return false;
  std::string s;
  if (!std::getline(f, s)) return false;
  size_t i = 0;
  while (i < s.size() && (s[i] == ' ' || s[i] == '\t')) ++i;
  if (i >= s.size() || s[i] < '0' || s[i] > '9') return false;
  *n = std::strtoull(s.c_str() + i, nullptr, 10);
  return true;
}

int main(int argc, char** argv) {
  std::vector<const char*> pos;
  const char* config = nullptr;
  int device = 0;
  bool sorted = false;
  bool check = false;
  for (int i = 1; i < argc; ++i) {
    if (!std::strcmp(argv[i], "--config") && i + 1 < argc) {
      config = argv[++i];
    } else if (!std::strcmp(argv[i], "--device") && i + 1 < argc) {
      device = std::atoi(argv[++i]);
    } else if (!std::strcmp(argv[i], "--sorted")) {
      sorted = true;
    } else if (!std::strcmp(argv[i], "--check")) {
      check = true;
    } else {
      pos.push_back(argv[i]);
    }
  }
  if (pos.size() != 4) {
    std::printf("You input %d args\n", argc);
    std::fprintf(stderr, "Usage: %s <k-mer file> k l <output file> [--config <file>] [--device N] [--sorted] [--check]\n", argv[0]);
    return EXIT_FAILURE;
  }
  if (config && !check_config(config)) {
    std::fprintf(stderr, "Error: could not read config file %s\n", config);
    return EXIT_FAILURE;
  }
  const int k = std::atoi(pos[1]);
  const int l = std::atoi(pos[2]);
  if (check) {
    unsigned long long n = 0;
    if (!check_input(pos[0], &n)) {
      std::fprintf(stderr, "Error: %s has no k-mer count line\n", pos[0]);
      return EXIT_FAILURE;
    }
    if (k < 2 || k > 63 || l < 1 || l > 16 || l > k - 1) {
      std::fprintf(stderr, "Error: need 2 <= k <= 63 and 1 <= l <= min(16, k-1)\n");
      return EXIT_FAILURE;
    }
    std::printf("ok: %llu k-mers, k = %d, l = %d%s%s\n", n, k, l, config ? ", config " : "", config ? config : "");
    return 0;
  }
  uc_ctx* ctx = nullptr;
  uc_status s = uc_ctx_create(device, 0, &ctx);
  if (s != UC_OK) {
    std::fprintf(stderr, "Error: %s\n", uc_status_str(s));
    return EXIT_FAILURE;
  }
  if (sorted) uc_ctx_set_sorted_output(ctx, 1);
  uc_stats st{};
  const auto t0 = std::chrono::steady_clock::now();
  s = uc_compact_file(ctx, pos[0], k, l, pos[3], &st);
  const double total_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (s != UC_OK) {
    std::fprintf(stderr, "Error: %s: %s\n", uc_status_str(s), uc_last_error(ctx));
    uc_ctx_destroy(ctx);
    return EXIT_FAILURE;
  }
  std::printf("kmer size: %llu, kmers: %llu\n", (unsigned long long)st.n_kmers * (unsigned long long)k,
              (unsigned long long)st.n_kmers);
  std::printf("kmers: %llu, cross k-mers: %llu, tiles: %llu (%llu oversized), segments: %llu\n",
              (unsigned long long)st.n_kmers, (unsigned long long)st.n_cross, (unsigned long long)st.n_tiles,
              (unsigned long long)st.n_big_tiles, (unsigned long long)st.n_segments);
  std::printf("Time to pack and bucket by l-minimizers: %.3fs\n", (st.ms_pack + st.ms_bucket) / 1e3);
  std::printf("Time to assemble and compact tiles: %.3fs\n", st.ms_tiles / 1e3);
  std::printf("Time to stitch cross-tile unitigs: %.3fs\n", st.ms_stitch / 1e3);
  std::printf("Device time: %.3fs\n", st.ms_total / 1e3);
  std::printf("Total time: %.3fs\n", total_s);
  uc_ctx_destroy(ctx);
  return 0;
}
