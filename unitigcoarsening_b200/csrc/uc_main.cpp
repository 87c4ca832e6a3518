// uc_main — command-line driver with the reference's interface:
//
//   uc_main <k-mer file> k l <output file> [--config <file>] [--device N] [--sorted]
//
// (driver.cpp:422-432: exactly four positional arguments, no defaults).  The
// unitig lines are appended to the output file as the reference does
// (compact.h:10,25).  The reference ships three config files (base_config.txt,
// cond_config.txt, fourpart_config.txt) that none of its code reads; --config
// accepts them, checks that they parse (seven lines of numbers and a final
// word), and changes nothing.  Phase times are printed like the reference's
// timers (driver.cpp:641-657).  --sorted writes the lines in byte order, so
// that equal input gives byte-equal output.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "uc.h"

static bool check_config(const char* path) {
  std::ifstream f(path);
  if (!f.is_open()) return false;
  std::vector<std::string> lines;
  std::string s;
  while (std::getline(f, s)) lines.push_back(s);
  if (lines.empty()) return false;
  for (size_t i = 0; i + 1 < lines.size(); ++i) {
    char* end = nullptr;
    std::strtod(lines[i].c_str(), &end);
    if (end == lines[i].c_str()) return false;
  }
  return true;
}

int main(int argc, char** argv) {
  std::vector<const char*> pos;
  const char* config = nullptr;
  int device = 0;
  bool sorted = false;
  for (int i = 1; i < argc; ++i) {
    if (!std::strcmp(argv[i], "--config") && i + 1 < argc) {
      config = argv[++i];
    } else if (!std::strcmp(argv[i], "--device") && i + 1 < argc) {
      device = std::atoi(argv[++i]);
    } else if (!std::strcmp(argv[i], "--sorted")) {
      sorted = true;
    } else {
      pos.push_back(argv[i]);
    }
  }
  if (pos.size() != 4) {
    std::printf("You input %d args\n", argc);
    std::fprintf(stderr, "Usage: %s <k-mer file> k l <output file> [--config <file>] [--device N] [--sorted]\n", argv[0]);
    return EXIT_FAILURE;
  }
  if (config && !check_config(config)) {
    std::fprintf(stderr, "Error: could not read config file %s\n", config);
    return EXIT_FAILURE;
  }
  const int k = std::atoi(pos[1]);
  const int l = std::atoi(pos[2]);
  uc_ctx* ctx = nullptr;
  uc_status s = uc_ctx_create(device, 0, &ctx);
  if (s != UC_OK) {
    std::fprintf(stderr, "Error: %s\n", uc_status_str(s));
    return EXIT_FAILURE;
  }
  if (sorted) uc_ctx_set_sorted_output(ctx, 1);
  uc_stats st{};
  s = uc_compact_file(ctx, pos[0], k, l, pos[3], &st);
  if (s != UC_OK) {
    std::fprintf(stderr, "Error: %s: %s\n", uc_status_str(s), uc_last_error(ctx));
    uc_ctx_destroy(ctx);
    return EXIT_FAILURE;
  }
  std::printf("kmers: %llu, cross k-mers: %llu, tiles: %llu (%llu oversized), segments: %llu\n",
              (unsigned long long)st.n_kmers, (unsigned long long)st.n_cross, (unsigned long long)st.n_tiles,
              (unsigned long long)st.n_big_tiles, (unsigned long long)st.n_segments);
  std::printf("Time to pack and bucket by l-minimizers: %.3fs\n", (st.ms_pack + st.ms_bucket) / 1e3);
  std::printf("Time to assemble and compact tiles: %.3fs\n", st.ms_tiles / 1e3);
  std::printf("Time to stitch cross-tile unitigs: %.3fs\n", st.ms_stitch / 1e3);
  std::printf("Device time: %.3fs\n", st.ms_total / 1e3);
  uc_ctx_destroy(ctx);
  return 0;
}
