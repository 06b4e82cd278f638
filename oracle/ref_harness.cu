// ref_harness.cu -- drives the reference G-LeCo implementation, compiled from the reference's
// own headers (include path -I<reference tree>), to pin the oracle.  TEST INFRASTRUCTURE ONLY.
//
// Modes (all file I/O is raw little-endian arrays):
//   partition  <dtype> <values.bin> <out.bin>
//        VariableLengthPartitioner<T>::partition() (compression/CpuPartitioner.cuh:342).
//        out.bin = int64 P, then P x {int32 start, int32 end, int32 bits}.
//   hostdecode <dtype> <blob.bin> <positions.bin> <out.bin> [repeat]
//        LeCoGPU<T>::createDirectAccessHandle(blob, size, false) + directRandomAccessCPU
//        (api/G-LeCo.cuh:1157, :1337): the reference's only host-side decoder.  Prints the
//        seconds per pass (best of `repeat`) on stdout.
//   hostdecode_all <dtype> <blob.bin> <values.bin> <threads> <repeat> [mism.bin]
//        createDirectAccessHandle(blob, size, false) + directRandomAccessCPU over EVERY position
//        of the column, split into <threads> contiguous slices decoded by as many host threads
//        (the function only reads the handle, so the threads share it).  Prints one line
//        "pass <seconds>" per pass over all positions (wall clock), then the best seconds and the
//        number of values that differ from values.bin; mism.bin (optional) receives those
//        positions as int64.
//   golden     <dtype> <values.bin> <outprefix> <fixed|var|v6>
//        GPU only: LeCoGPU<T>::compress (api/G-LeCo.cuh:349, stock fixed TILE_SIZE=4096 path,
//        stock CPU-partitioner path, or the GPU-partitioner path use_gpu_partitioning = true)
//        followed by the CPU serialize (api/G-LeCo.cuh:826).  Writes <outprefix>.blob and prints
//        the reported compressed size.  Only the reference's compression kernels run on the GPU;
//        none of its decoders does.
//   gpudecode  <dtype> <blob.bin> <values.bin> <repeat>
//        GPU only: deserializeGPU (api/G-LeCo.cuh:2157) of a blob, then the reference's own
//        full decoders decompressFullFile_BitPacked (:1739), _OnTheFly_Optimized_V2 (:1842) and
//        _WorkStealingAdvanced (:220), then deserializeGPU(blob, true) and
//        decompressFullFile_PreUnpacked (:1790), each `repeat` times; prints one line per decoder with the
//        best API-call seconds (output allocation, kernel, device-to-host copy, free) and the
//        values that differ from values.bin.  decompressFullFile_WorkStealing (:166) is not run:
//        its work counter is a fresh cudaMalloc that the kernel resets from one thread while the
//        other blocks may already read it, so an arbitrary start value can index outside the
//        partition arrays.  The decoders read the word after a field, one past the bitstream at
//        its end; the run is refused when the bitstream ends exactly at a 2 MB boundary, where
//        that word would fall outside the allocation's pages.
//   gpura      <dtype> <blob.bin> <positions.bin> <values.bin> <partition_len> <repeat>
//        GPU only: deserializeGPU of a blob, then the reference's own randomAccessFixed (:1878,
//        partition = pos / len; skipped when partition_len <= 0, for variable partitions) and
//        decompress (:615, binary search over the partitions), each `repeat` times over the
//        int32 positions; prints one line per method
//        with the best API-call seconds and the lookups that differ from values[pos].  The same
//        2 MB-boundary rule as gpudecode applies.  With [outprefix] the column is also
//        deserialized with preUnpackDeltas = true and randomAccessPreUnpacked (:696) and
//        randomAccessFixedPreUnpacked (:1931) answer the same positions; every method's output is
//        written to <outprefix>.<method>.bin.  (randomAccessPreUnpacked answers at most
//        SMs x 32 x 256 positions, randomAccessFixedPreUnpacked SMs x 32 x 512: neither kernel
//        has a grid-stride loop.)
//   gpucompress <dtype> <values.bin> <fixed|v6|var> <repeat>
//        GPU only: the reference's own LeCoGPU<T>::compress (api/G-LeCo.cuh:349) with fixed
//        partitions of TILE_SIZE, with its GPU partitioner (use_gpu_partitioning = true) or with
//        its CPU partitioner (use_variable_partitioning = true, the default variable mode), each
//        `repeat` times; prints the best API-call seconds (host values in, the upload included)
//        and the reported compressed size.
//   v6         <dtype> <values.bin> <out.bin>
//        GPU only: GPUVariableLengthPartitionerV6<T>(values, 2048).partition()
//        (compression/GpuPartitioner.cuh:34-214, base size as compress passes it).  out.bin as for
//        `partition`; prints the seconds partition() took (the upload excluded).
//
// Without a CUDA device (this harness is also run in CPU-only containers) the CUDA stream
// calls made by the LeCoGPU constructor/destructor are answered by ref_stubs.cpp when
// GLC_REF_CPU_ONLY=1, because directRandomAccessCPU uses no device state.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <chrono>
#include <thread>
#include <vector>
#include <string>
#include "api/G-LeCo.cuh"

static std::vector<uint8_t> read_file(const char* path) {
  std::vector<uint8_t> b;
  FILE* f = fopen(path, "rb");
  if (!f) { fprintf(stderr, "cannot open %s\n", path); exit(2); }
  fseek(f, 0, SEEK_END); long n = ftell(f); fseek(f, 0, SEEK_SET);
  b.resize((size_t)n);
  if (n > 0 && fread(b.data(), 1, (size_t)n, f) != (size_t)n) { fprintf(stderr, "short read %s\n", path); exit(2); }
  fclose(f);
  return b;
}

static void write_file(const char* path, const void* p, size_t n) {
  FILE* f = fopen(path, "wb");
  if (!f) { fprintf(stderr, "cannot write %s\n", path); exit(2); }
  if (n > 0) fwrite(p, 1, n, f);
  fclose(f);
}

template <typename T> static std::vector<T> as_vec(const std::vector<uint8_t>& b) {
  std::vector<T> v(b.size() / sizeof(T));
  if (!v.empty()) memcpy(v.data(), b.data(), v.size() * sizeof(T));
  return v;
}

template <typename T> static int run_partition(const char* in, const char* out) {
  std::vector<T> v = as_vec<T>(read_file(in));
  VariableLengthPartitioner<T> vp(v, SPLIT_THRESHOLD, MIN_PARTITION_SIZE, "");
  std::vector<PartitionInfo> parts = vp.partition();
  std::vector<uint8_t> o(8 + parts.size() * 12);
  int64_t P = (int64_t)parts.size();
  memcpy(o.data(), &P, 8);
  for (size_t i = 0; i < parts.size(); i++) {
    int32_t rec[3] = {parts[i].start_idx, parts[i].end_idx, parts[i].delta_bits};
    memcpy(o.data() + 8 + 12 * i, rec, 12);
  }
  write_file(out, o.data(), o.size());
  return 0;
}

template <typename T> static int run_hostdecode(const char* blobp, const char* posp, const char* out, int repeat) {
  std::vector<uint8_t> blob = read_file(blobp);
  std::vector<int> pos = as_vec<int>(read_file(posp));
  LeCoGPU<T> codec;
  DirectAccessHandle<T>* h = codec.createDirectAccessHandle(blob.data(), blob.size(), false);
  if (!h) { fprintf(stderr, "createDirectAccessHandle rejected the blob\n"); return 3; }
  std::vector<T> res;
  double best = 1e30;
  for (int r = 0; r < (repeat > 0 ? repeat : 1); r++) {
    auto t0 = std::chrono::steady_clock::now();
    codec.directRandomAccessCPU(h, pos, res, false);
    auto t1 = std::chrono::steady_clock::now();
    double s = std::chrono::duration<double>(t1 - t0).count();
    if (s < best) best = s;
  }
  write_file(out, res.data(), res.size() * sizeof(T));
  printf("%.9f\n", best);
  h->~DirectAccessHandle<T>();
  free(h);
  return 0;
}

template <typename T> static int run_hostdecode_all(const char* blobp, const char* valp, int threads, int repeat,
                                                    const char* mism_out) {
  std::vector<uint8_t> blob = read_file(blobp);
  std::vector<T> want = as_vec<T>(read_file(valp));
  LeCoGPU<T> codec;
  DirectAccessHandle<T>* h = codec.createDirectAccessHandle(blob.data(), blob.size(), false);
  if (!h) { fprintf(stderr, "createDirectAccessHandle rejected the blob\n"); return 3; }
  const int64_t n = (int64_t)want.size();
  if (threads < 1) threads = 1;
  std::vector<std::vector<int>> pos(threads);
  std::vector<std::vector<T>> out(threads);
  std::vector<int64_t> first(threads + 1);
  for (int t = 0; t <= threads; t++) first[t] = n * t / threads;
  for (int t = 0; t < threads; t++) {
    pos[t].resize((size_t)(first[t + 1] - first[t]));
    for (int64_t i = first[t]; i < first[t + 1]; i++) pos[t][(size_t)(i - first[t])] = (int)i;
  }
  double best = 1e30;
  for (int r = 0; r < (repeat > 0 ? repeat : 1); r++) {
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> th;
    for (int t = 0; t < threads; t++)
      th.emplace_back([&, t] { codec.directRandomAccessCPU(h, pos[t], out[t], false); });
    for (auto& x : th) x.join();
    auto t1 = std::chrono::steady_clock::now();
    const double sec = std::chrono::duration<double>(t1 - t0).count();
    printf("pass %.9f\n", sec);
    fflush(stdout);
    best = std::min(best, sec);
  }
  std::vector<int64_t> bad;
  for (int t = 0; t < threads; t++) {
    if ((int64_t)out[t].size() != first[t + 1] - first[t]) { fprintf(stderr, "short output\n"); return 3; }
    for (int64_t i = first[t]; i < first[t + 1]; i++)
      if (out[t][(size_t)(i - first[t])] != want[(size_t)i]) bad.push_back(i);
  }
  if (mism_out) write_file(mism_out, bad.data(), bad.size() * sizeof(int64_t));
  printf("%.9f %zu\n", best, bad.size());
  h->~DirectAccessHandle<T>();
  free(h);
  return 0;
}

template <typename T> static int run_v6(const char* in, const char* out) {
  std::vector<T> v = as_vec<T>(read_file(in));
  GPUVariableLengthPartitionerV6<T> vp(v, 2048, 0);
  cudaDeviceSynchronize();  // the constructor's upload is not part of partition()
  auto t0 = std::chrono::steady_clock::now();
  std::vector<PartitionInfo> parts = vp.partition();
  auto t1 = std::chrono::steady_clock::now();
  printf("%.9f\n", std::chrono::duration<double>(t1 - t0).count());
  std::vector<uint8_t> o(8 + parts.size() * 12);
  int64_t P = (int64_t)parts.size();
  memcpy(o.data(), &P, 8);
  for (size_t i = 0; i < parts.size(); i++) {
    int32_t rec[3] = {parts[i].start_idx, parts[i].end_idx, parts[i].delta_bits};
    memcpy(o.data() + 8 + 12 * i, rec, 12);
  }
  write_file(out, o.data(), o.size());
  return 0;
}

template <typename T> static int run_gpudecode(const char* blobp, const char* valp, int repeat) {
  std::vector<uint8_t> blob = read_file(blobp);
  std::vector<T> want = as_vec<T>(read_file(valp));
  if (blob.size() < sizeof(SerializedHeader)) { fprintf(stderr, "short blob\n"); return 3; }
  SerializedHeader hdr;
  memcpy(&hdr, blob.data(), sizeof hdr);
  const uint64_t dbytes = ((hdr.delta_array_size_bytes + 3) / 4) * 4;
  if (dbytes == 0 || dbytes % (2u << 20) == 0) {
    fprintf(stderr, "bitstream ends at a 2 MB boundary: not run\n");
    return 4;
  }
  LeCoGPU<T> codec;
  SerializedData sd;
  sd.data = new uint8_t[blob.size()];
  memcpy(sd.data, blob.data(), blob.size());
  sd.size = blob.size();
  CompressedData<T>* cd = codec.deserializeGPU(&sd, false);
  if (!cd) { fprintf(stderr, "deserializeGPU rejected the blob\n"); return 3; }
  typedef void (LeCoGPU<T>::*Dec)(CompressedData<T>*, std::vector<T>&);
  const struct { const char* name; Dec f; } decs[] = {
      {"decompressFullFile_BitPacked", &LeCoGPU<T>::decompressFullFile_BitPacked},
      {"decompressFullFile_OnTheFly_Optimized_V2", &LeCoGPU<T>::decompressFullFile_OnTheFly_Optimized_V2},
      {"decompressFullFile_WorkStealingAdvanced", &LeCoGPU<T>::decompressFullFile_WorkStealingAdvanced}};
  for (const auto& d : decs) {
    std::vector<T> out;
    double best = 1e30;
    for (int r = 0; r < (repeat > 0 ? repeat : 1); r++) {
      cudaDeviceSynchronize();
      auto t0 = std::chrono::steady_clock::now();
      (codec.*(d.f))(cd, out);
      auto t1 = std::chrono::steady_clock::now();
      best = std::min(best, std::chrono::duration<double>(t1 - t0).count());
    }
    size_t bad = out.size() == want.size() ? 0 : want.size();
    for (size_t i = 0; i < out.size() && i < want.size(); i++) bad += out[i] != want[i];
    printf("%s %.9f %zu\n", d.name, best, bad);
  }
  codec.cleanup(cd);
  CompressedData<T>* cu = codec.deserializeGPU(&sd, true);
  if (!cu) { fprintf(stderr, "deserializeGPU(preUnpackDeltas) rejected the blob\n"); return 3; }
  {
    std::vector<T> out;
    double best = 1e30;
    for (int r = 0; r < (repeat > 0 ? repeat : 1); r++) {
      cudaDeviceSynchronize();
      auto t0 = std::chrono::steady_clock::now();
      codec.decompressFullFile_PreUnpacked(cu, out);
      auto t1 = std::chrono::steady_clock::now();
      best = std::min(best, std::chrono::duration<double>(t1 - t0).count());
    }
    size_t bad = out.size() == want.size() ? 0 : want.size();
    for (size_t i = 0; i < out.size() && i < want.size(); i++) bad += out[i] != want[i];
    printf("decompressFullFile_PreUnpacked %.9f %zu\n", best, bad);
  }
  codec.cleanup(cu);
  return 0;
}

template <typename T> static int run_gpura(const char* blobp, const char* posp, const char* valp, int plen,
                                           int repeat, const char* outprefix) {
  std::vector<uint8_t> blob = read_file(blobp);
  std::vector<int> pos = as_vec<int>(read_file(posp));
  std::vector<T> vals = as_vec<T>(read_file(valp));
  if (blob.size() < sizeof(SerializedHeader)) { fprintf(stderr, "short blob\n"); return 3; }
  SerializedHeader hdr;
  memcpy(&hdr, blob.data(), sizeof hdr);
  const uint64_t dbytes = ((hdr.delta_array_size_bytes + 3) / 4) * 4;
  if (dbytes == 0 || dbytes % (2u << 20) == 0) {
    fprintf(stderr, "bitstream ends at a 2 MB boundary: not run\n");
    return 4;
  }
  for (int p : pos)
    if (p < 0 || (size_t)p >= vals.size()) { fprintf(stderr, "position outside the column\n"); return 3; }
  LeCoGPU<T> codec;
  SerializedData sd;
  sd.data = new uint8_t[blob.size()];
  memcpy(sd.data, blob.data(), blob.size());
  sd.size = blob.size();
  CompressedData<T>* cd = codec.deserializeGPU(&sd, false);
  if (!cd) { fprintf(stderr, "deserializeGPU rejected the blob\n"); return 3; }
  for (int m = 0; m < 2; m++) {
    if (m == 0 && plen <= 0) continue;  // variable partitions: no fixed-length method
    std::vector<T> out;
    double best = 1e30;
    for (int r = 0; r < (repeat > 0 ? repeat : 1); r++) {
      cudaDeviceSynchronize();
      auto t0 = std::chrono::steady_clock::now();
      if (m == 0) codec.randomAccessFixed(cd, pos, out, plen);
      else codec.decompress(cd, pos, out);
      auto t1 = std::chrono::steady_clock::now();
      best = std::min(best, std::chrono::duration<double>(t1 - t0).count());
    }
    size_t bad = out.size() == pos.size() ? 0 : pos.size();
    for (size_t i = 0; i < out.size() && i < pos.size(); i++) bad += out[i] != vals[pos[i]];
    const char* name = m == 0 ? "randomAccessFixed" : "decompress";
    printf("%s %.9f %zu\n", name, best, bad);
    if (outprefix) write_file((std::string(outprefix) + "." + name + ".bin").c_str(), out.data(), out.size() * sizeof(T));
  }
  codec.cleanup(cd);
  if (!outprefix) return 0;
  CompressedData<T>* cu = codec.deserializeGPU(&sd, true);
  if (!cu) { fprintf(stderr, "deserializeGPU(preUnpackDeltas) rejected the blob\n"); return 3; }
  for (int m = 0; m < 2; m++) {
    if (m == 1 && plen <= 0) continue;
    std::vector<T> out;
    double best = 1e30;
    for (int r = 0; r < (repeat > 0 ? repeat : 1); r++) {
      cudaDeviceSynchronize();
      auto t0 = std::chrono::steady_clock::now();
      if (m == 0) codec.randomAccessPreUnpacked(cu, pos, out);
      else codec.randomAccessFixedPreUnpacked(cu, pos, out, plen);
      auto t1 = std::chrono::steady_clock::now();
      best = std::min(best, std::chrono::duration<double>(t1 - t0).count());
    }
    size_t bad = out.size() == pos.size() ? 0 : pos.size();
    for (size_t i = 0; i < out.size() && i < pos.size(); i++) bad += out[i] != vals[pos[i]];
    const char* name = m == 0 ? "randomAccessPreUnpacked" : "randomAccessFixedPreUnpacked";
    printf("%s %.9f %zu\n", name, best, bad);
    write_file((std::string(outprefix) + "." + name + ".bin").c_str(), out.data(), out.size() * sizeof(T));
  }
  codec.cleanup(cu);
  return 0;
}

template <typename T> static int run_gpucompress(const char* in, const std::string& how, int repeat) {
  const bool v6 = how == "v6", var = how != "fixed";
  std::vector<T> v = as_vec<T>(read_file(in));
  LeCoGPU<T> codec;
  double best = 1e30;
  long long size = 0;
  for (int r = 0; r < (repeat > 0 ? repeat : 1); r++) {
    cudaDeviceSynchronize();
    auto t0 = std::chrono::steady_clock::now();
    CompressedData<T>* cd = codec.compress(v, var, &size, v6, "");
    cudaDeviceSynchronize();
    auto t1 = std::chrono::steady_clock::now();
    if (!cd) { fprintf(stderr, "compress returned null\n"); return 3; }
    best = std::min(best, std::chrono::duration<double>(t1 - t0).count());
    codec.cleanup(cd);
  }
  printf("compress_%s %.9f %lld\n", how.c_str(), best, size);
  return 0;
}

template <typename T> static int run_golden(const char* in, const char* prefix, bool var, bool gpu_part) {
  std::vector<T> v = as_vec<T>(read_file(in));
  LeCoGPU<T> codec;
  long long size = 0;
  CompressedData<T>* cd = codec.compress(v, var, &size, gpu_part, "");
  if (!cd) { fprintf(stderr, "compress returned null\n"); return 3; }
  SerializedData* sd = codec.serialize(cd);
  if (!sd) { fprintf(stderr, "serialize returned null\n"); return 3; }
  std::string bp = std::string(prefix) + ".blob";
  write_file(bp.c_str(), sd->data, sd->size);
  printf("%lld\n", size);
  delete sd;
  codec.cleanup(cd);
  return 0;
}

template <typename T> static int dispatch(int argc, char** argv) {
  std::string mode = argv[1];
  if (mode == "partition" && argc >= 5) return run_partition<T>(argv[3], argv[4]);
  if (mode == "hostdecode" && argc >= 6) return run_hostdecode<T>(argv[3], argv[4], argv[5], argc >= 7 ? atoi(argv[6]) : 1);
  if (mode == "golden" && argc >= 6) {
    const std::string how = argv[5];
    return run_golden<T>(argv[3], argv[4], how != "fixed", how == "v6");
  }
  if (mode == "v6" && argc >= 5) return run_v6<T>(argv[3], argv[4]);
  if (mode == "gpucompress" && argc >= 6) return run_gpucompress<T>(argv[3], argv[4], atoi(argv[5]));
  if (mode == "hostdecode_all" && argc >= 7)
    return run_hostdecode_all<T>(argv[3], argv[4], atoi(argv[5]), atoi(argv[6]), argc >= 8 ? argv[7] : nullptr);
  if (mode == "gpudecode" && argc >= 6) return run_gpudecode<T>(argv[3], argv[4], atoi(argv[5]));
  if (mode == "gpura" && argc >= 8)
    return run_gpura<T>(argv[3], argv[4], argv[5], atoi(argv[6]), atoi(argv[7]), argc >= 9 ? argv[8] : nullptr);
  fprintf(stderr, "bad arguments\n");
  return 2;
}

int main(int argc, char** argv) {
  if (argc < 3) { fprintf(stderr, "usage: ref_harness <mode> <i32|i64|u64|u32> ...\n"); return 2; }
  std::string dt = argv[2];
  if (dt == "i32") return dispatch<int>(argc, argv);
  if (dt == "i64") return dispatch<long long>(argc, argv);
  if (dt == "u64") return dispatch<unsigned long long>(argc, argv);
  if (dt == "u32") return dispatch<unsigned int>(argc, argv);
  fprintf(stderr, "unknown dtype %s\n", dt.c_str());
  return 2;
}
