// Driver for the reference's own codec and hash, compiled from the reference sources
// where they lie (see build_ref.sh; nothing of the reference is copied here). It writes
// golden vectors used to pin the oracle and the product's segment writer/decoders:
//   ref_driver codec <dir>   segment files written by pfor_compress /
//                            pfor_delta_compress (compress.cu:271-527) for seeded value
//                            sets, each with the values pfor_decompress (compress.cu:180)
//                            reads back
//   ref_driver murmur <file> MurmurHash64A (MurmurHash2_64.cu:201) of seeded byte strings
//   ref_driver like <file>   the reference's LIKE matcher (struct gpu_regex, filter.cu:67-129)
//                            over a fixed set of dictionary entries and patterns
#include REF_COMPRESS_CU
#ifdef REF_GPU_REGEX
#include REF_GPU_REGEX
#endif

#include <cstdint>
#include <cstdio>
#include <fstream>
#include <vector>

thrust::device_vector<unsigned char> scratch;
map<string, unsigned int> cpy_bits;
map<string, long long int> cpy_init_val;
bool delta = false;
size_t int_size = sizeof(long long int);
size_t float_size = sizeof(double);

uint64_t MurmurHash64A(const void* key, int len, unsigned int seed);

static uint64_t lcg_state = 12345;
static uint64_t next_u64() {
  lcg_state = lcg_state * 6364136223846793005ULL + 1442695040888963407ULL;
  return lcg_state >> 11;
}
static long long rnd(long long lo, long long hi) { return lo + (long long)(next_u64() % (uint64_t)(hi - lo + 1)); }

struct Case {
  const char* name;
  bool use_delta;
  std::vector<long long> v;
};

static std::vector<Case> cases() {
  std::vector<Case> c;
  auto add = [&](const char* n, bool d, std::vector<long long> v) { c.push_back({n, d, std::move(v)}); };
  std::vector<long long> v;
  v.clear(); for (int i = 0; i < 1000; i++) v.push_back(rnd(5000, 5200)); add("for8", false, v);
  v.clear(); for (int i = 0; i < 1000; i++) v.push_back(rnd(0, 60000)); add("for16", false, v);
  v.clear(); for (int i = 0; i < 1000; i++) v.push_back(rnd(-1000000, 100000000)); add("for32", false, v);
  v.clear(); for (int i = 0; i < 777; i++) v.push_back(rnd(-(1LL << 40), 1LL << 41)); add("for64", false, v);
  v.assign(333, 7); add("const", false, v);
  v.clear(); for (int i = 0; i < 1001; i++) v.push_back(rnd(19920101, 19981231)); add("dates16", false, v);
  long long x = 100;
  v.clear(); for (int i = 0; i < 1500; i++) { x += rnd(0, 9); v.push_back(x); } add("delta_small", true, v);
  x = -5000;
  v.clear(); for (int i = 0; i < 900; i++) { x += rnd(1, 1 << 20); v.push_back(x); } add("delta_wide", true, v);
  v.assign(1, 42); add("delta_single", true, v);
  x = 0;
  v.clear(); for (int i = 0; i < 1234; i++) { x += rnd(0, 1) * 4; v.push_back(x); } add("delta_dups", true, v);
  v.clear(); for (int i = 0; i < 500; i++) v.push_back(rnd(0, 100)); add("delta_unsorted", true, v);
  return c;
}

static int do_codec(const std::string& dir) {
  for (auto& cs : cases()) {
    delta = cs.use_delta;
    std::vector<long long> work(cs.v);
    thrust::host_vector<long long, pinned_allocator<long long> > host(work.size() + 16);
    std::string f = dir + "/" + cs.name + ".seg";
    curr_file = f;
    pfor_compress(work.data(), work.size() * sizeof(long long), f, host, false);
    // read back with the reference decoder
    std::ifstream in(f, std::ios::binary);
    std::vector<char> img((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    std::vector<long long> out(cs.v.size() + 16);
    unsigned int d_v[4];
    long long s_v[2];
    size_t n = pfor_decompress(out.data(), img.data(), d_v, s_v, std::string(cs.name));
    if (n != cs.v.size()) {
      std::fprintf(stderr, "%s: decoded %zu of %zu\n", cs.name, n, cs.v.size());
      return 1;
    }
    std::ofstream vo(dir + "/" + cs.name + ".values", std::ios::binary);
    vo.write((const char*)cs.v.data(), cs.v.size() * 8);
    std::ofstream dout(dir + "/" + cs.name + ".decoded", std::ios::binary);
    dout.write((const char*)out.data(), n * 8);
  }
  return 0;
}

static int do_murmur(const std::string& path) {
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return 1;
  for (int len = 0; len <= 40; len++) {
    for (int rep = 0; rep < 3; rep++) {
      std::vector<unsigned char> b(len);
      for (auto& c : b) c = (unsigned char)(next_u64() & 0xff);
      unsigned int seed = rep == 2 ? 0 : 100;
      uint64_t h = MurmurHash64A(b.data(), len, seed);
      std::fprintf(f, "%u ", seed);
      for (auto c : b) std::fprintf(f, "%02x", c);
      std::fprintf(f, "%s %llu\n", len ? "" : "-", (unsigned long long)h);
    }
  }
  std::fclose(f);
  return 0;
}

#ifdef REF_GPU_REGEX
// Entries of a char column of width 12 (NUL padded; one fills the width) and LIKE
// patterns shorter than the width, as filter.cu passes them: the entries back to back,
// the pattern in a zeroed buffer of the column width, len = {width}.
static int do_like(const std::string& path) {
  const unsigned int width = 12;
  const char* entries[] = {"AUTOMOBILE", "BUILDING", "FURNITURE", "HOUSEHOLD", "MACHINERY", "A.B", "A.BC",
                           "ABC", "abc.def", "%PCT", "100%", "", "X", "XYZXYZXYZXYZ", "..", "a_b", "AAB",
                           "ABAB", "MACHINE.RY", "ABABABABABA", "BA", "AXBXC"};
  const char* patterns[] = {"%", "%%", "", "A%", "%A", "%A%", "A?C", "A?B", "???", "?%", "%?", "%.%",
                            "%B%I%", "BUILDING", "BUILDING%", "BUILD", "%ING", "%Y", "_", "a_b", "X%Z",
                            "XYZ%XYZ", "%XYZ", "?.?", "A%B%", "%AB", "A%%B", "100%", "%PCT", "%%PCT", "M%Y",
                            "MACHINE%RY", "M?CHINE.RY", "%BA", "%ABA", "A%C", "%B%C", "?B%", "AB?B", "%?%?"};
  const size_t ne = sizeof(entries) / sizeof(entries[0]), np = sizeof(patterns) / sizeof(patterns[0]);
  std::vector<char> src(ne * width, 0);
  for (size_t i = 0; i < ne; i++) std::memcpy(&src[i * width], entries[i], std::min<size_t>(width, std::strlen(entries[i])));
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return 1;
  std::fprintf(f, "width %u\n", width);
  for (size_t i = 0; i < ne; i++) {
    std::fprintf(f, "entry ");
    for (unsigned int k = 0; k < width; k++) std::fprintf(f, "%02x", (unsigned char)src[i * width + k]);
    std::fprintf(f, "\n");
  }
  for (size_t j = 0; j < np; j++) {
    std::vector<char> pat(width, 0);
    std::memcpy(pat.data(), patterns[j], std::strlen(patterns[j]));
    std::vector<char> dest(ne, 0);
    unsigned int len = width;
    gpu_regex m(src.data(), pat.data(), (bool*)dest.data(), &len);
    for (size_t i = 0; i < ne; i++) m(i);
    std::fprintf(f, "pattern %s ", std::strlen(patterns[j]) ? "" : "-");
    for (size_t k = 0; k < std::strlen(patterns[j]); k++) std::fprintf(f, "%02x", (unsigned char)patterns[j][k]);
    std::fprintf(f, " ");
    for (size_t i = 0; i < ne; i++) std::fprintf(f, "%d", dest[i] ? 1 : 0);
    std::fprintf(f, "\n");
  }
  std::fclose(f);
  return 0;
}
#endif

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  std::string mode = argv[1];
  if (mode == "codec") return do_codec(argv[2]);
  if (mode == "murmur") return do_murmur(argv[2]);
#ifdef REF_GPU_REGEX
  if (mode == "like") return do_like(argv[2]);
#endif
  return 2;
}
