// A caller written the way the reference's driver (app/Main.cu) uses LeCoGPU<T>, compiled
// against include/glc_leco.hpp and libglc.so.  Exits 0 when every path returns the input.
#include <cstdio>
#include <random>
#include <vector>

#include "glc_leco.hpp"

template <typename T>
static int run(const char* name, const std::vector<T>& data) {
  LeCoGPU<T> codec;
  int bad = 0;
  std::mt19937_64 rng(7);
  std::vector<int> pos(10000);
  for (auto& p : pos) p = (int)(rng() % data.size());
  for (int var = 0; var < 2; var++) {
    long long size = 0;
    CompressedData<T>* cd = codec.compress(data, var == 1, &size);
    if (!cd || size <= 0) { printf("%s: compress failed\n", name); return 1; }
    std::vector<T> out;
    codec.decompressFullFile(cd, out);
    bad += out != data;
    codec.decompressFullFile_WorkStealing(cd, out);
    bad += out != data;
    codec.decompress(cd, pos, out);
    for (size_t k = 0; k < pos.size(); k++) bad += out[k] != data[pos[k]];
    if (!var) {
      codec.randomAccessFixed(cd, pos, out, 4096);
      for (size_t k = 0; k < pos.size(); k++) bad += out[k] != data[pos[k]];
      codec.decompressFullFile_Fix(cd, out, 4096);
      bad += out != data;
    }
    SerializedData* sd = codec.serializeGPU(cd);
    CompressedData<T>* back = codec.deserializeGPU(sd, true);
    if (!back) { printf("%s: deserialize failed\n", name); return 1; }
    codec.decompressFullFile(back, out);
    bad += out != data;
    codec.randomAccessPreUnpacked(back, pos, out);
    for (size_t k = 0; k < pos.size(); k++) bad += out[k] != data[pos[k]];
    DirectAccessHandle<T>* h = codec.createDirectAccessHandle(sd->data, sd->size, true);
    codec.directRandomAccessGPU(h, pos, out);
    for (size_t k = 0; k < pos.size(); k++) bad += out[k] != data[pos[k]];
    codec.destroyDirectAccessHandle(h);
    // a corrupted blob is rejected with nullptr, as in the reference
    sd->data[0] ^= 0xff;
    bad += codec.deserialize(sd) != nullptr;
    delete sd;
    codec.cleanup(back);
    codec.cleanup(cd);
  }
  printf("%s: %s\n", name, bad ? "MISMATCH" : "ok");
  return bad ? 1 : 0;
}

int main() {
  std::mt19937_64 rng(42);
  const int n = 1 << 20;
  std::vector<int> a(n);
  for (int i = 0; i < n; i++) a[i] = 1000 * i + (int)(rng() % 256);
  std::vector<long long> b(n);
  long long acc = 0;
  for (int i = 0; i < n; i++) { acc += (long long)(rng() % 2000); b[i] = acc; }
  std::vector<unsigned long long> c(n);
  for (int i = 0; i < n; i++) c[i] = (1ull << 40) + 977ull * i + (rng() % 4096);
  std::vector<unsigned int> d(n);
  for (int i = 0; i < n; i++) d[i] = 13u * i + (unsigned)(rng() % 100);
  int r = run("int", a) | run("long long", b) | run("unsigned long long", c) | run("unsigned int", d);
  return r;
}
