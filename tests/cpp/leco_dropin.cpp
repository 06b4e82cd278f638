// A caller written the way the reference's driver (app/Main.cu) uses LeCoGPU<T>, compiled
// against include/glc_leco.hpp and libglc.so.  Exits 0 when every path returns the input.
#include <cstdio>
#include <random>
#include <vector>

#include <cstdio>
#include <string>

#include "glc_io.hpp"
#include "glc_leco.hpp"

template <typename T>
static int run(const char* name, const std::vector<T>& data) {
  LeCoGPU<T> codec;
  int bad = 0;
  std::mt19937_64 rng(7);
  std::vector<int> pos(10000);
  for (auto& p : pos) p = (int)(rng() % data.size());
  for (int var = 0; var < 3; var++) {  // fixed, variable (CPU-partitioner model), variable (GPU partitioner)
    long long size = 0;
    CompressedData<T>* cd = codec.compress(data, var >= 1, &size, var == 2);
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

// The reference driver loads columns with read_binary_file / read_text_file (app/Main.cu:875-987).
template <typename T>
static int file_round_trip(const char* name, const std::vector<T>& data) {
  const std::string path = std::string("/tmp/glc_dropin_") + name + ".bin";
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) return 1;
  fwrite(data.data(), sizeof(T), data.size(), f);
  fclose(f);
  std::vector<T> loaded;
  if (!read_binary_file(path, loaded) || loaded != data) { printf("%s: read_binary_file failed\n", name); return 1; }
  LeCoGPU<T> codec;
  long long size = 0;
  CompressedData<T>* cd = codec.compress(loaded, true, &size);
  SerializedData* sd = codec.serialize(cd);
  const std::string blob = path + ".leco";
  int bad = !codec.saveToFile(sd->data, sd->size, blob);
  size_t bytes = 0;
  uint8_t* back = codec.loadFromFile(blob, bytes);
  bad += !back || bytes != sd->size;
  if (back) {
    SerializedData in;  // takes ownership of the loaded buffer
    in.data = back;
    in.size = bytes;
    CompressedData<T>* cd2 = codec.deserialize(&in);
    std::vector<T> out;
    if (cd2) codec.decompressFullFile(cd2, out);
    bad += !cd2 || out != data;
    if (cd2) codec.cleanup(cd2);
  }
  delete sd;
  codec.cleanup(cd);
  remove(path.c_str());
  remove(blob.c_str());
  printf("%s file round trip: %s\n", name, bad ? "MISMATCH" : "ok");
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
  r |= file_round_trip("int", a) | file_round_trip("ull", c);
  return r;
}
