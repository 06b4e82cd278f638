// glc_leco.hpp -- drop-in C++ class API of G-LeCo over the glc C ABI.
//
// Re-provides `template<typename T> class LeCoGPU` of the reference (api/G-LeCo.cuh:39-2304) with
// the same method names, signatures and ownership rules, plus the public types of
// api/G-LeCo_Types.cuh (ModelType, CompressedData<T>, SerializedData, DirectAccessHandle<T>).
// A caller written against the reference compiles unchanged against this header and libglc.so;
// every method runs the sm_100a kernels of libglc through include/glc.h.
//
// Error behaviour follows the reference's API: invalid input returns nullptr or clears the
// output vector (api/G-LeCo.cuh:168-177, :1020-1049); CUDA failures print and leave the output
// empty instead of calling exit().
#ifndef GLC_LECO_HPP_
#define GLC_LECO_HPP_

#include <cuda_runtime_api.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <new>
#include <string>
#include <type_traits>
#include <vector>

#include "glc.h"

// api/G-LeCo_Types.cuh:8-14
enum ModelType {
  MODEL_CONSTANT = 0,
  MODEL_LINEAR = 1,
  MODEL_POLYNOMIAL2 = 2,
  MODEL_POLYNOMIAL3 = 3,
  MODEL_DIRECT_COPY = 4
};

// api/G-LeCo_Types.cuh:18-42: the same device SoA fields, plus the owning glc column.
template <typename T>
struct CompressedData {
  int32_t* d_start_indices;
  int32_t* d_end_indices;
  int32_t* d_model_types;
  double* d_model_params;
  int32_t* d_delta_bits;
  int64_t* d_delta_array_bit_offsets;
  long long* d_error_bounds;
  uint32_t* delta_array;
  long long* d_plain_deltas;
  int num_partitions;
  int total_values;
  CompressedData<T>* d_self;
  glc_column* glc_col;  // owner of the arrays above
};

// api/G-LeCo_Types.cuh:45-72: move-only owner of a new[] host blob.
struct SerializedData {
  uint8_t* data;
  size_t size;
  SerializedData() : data(nullptr), size(0) {}
  ~SerializedData() { delete[] data; }
  SerializedData(const SerializedData&) = delete;
  SerializedData& operator=(const SerializedData&) = delete;
  SerializedData(SerializedData&& o) noexcept : data(o.data), size(o.size) { o.data = nullptr; o.size = 0; }
  SerializedData& operator=(SerializedData&& o) noexcept {
    if (this != &o) { delete[] data; data = o.data; size = o.size; o.data = nullptr; o.size = 0; }
    return *this;
  }
};

// api/G-LeCo_Types.cuh:75-107 (host view of a blob plus its device copy).  Random access on a
// handle runs on the device column built from the blob.
template <typename T>
struct DirectAccessHandle {
  const uint8_t* data_blob_host;
  size_t data_blob_size;
  glc_column* glc_col;
};

namespace glc_detail {
template <typename T> struct Code;
template <> struct Code<int> { static constexpr glc_dtype v = GLC_I32; };
template <> struct Code<long long> { static constexpr glc_dtype v = GLC_I64; };
template <> struct Code<long> { static constexpr glc_dtype v = GLC_I64; };
template <> struct Code<unsigned long long> { static constexpr glc_dtype v = GLC_U64; };
template <> struct Code<unsigned long> { static constexpr glc_dtype v = GLC_U64; };
template <> struct Code<unsigned int> { static constexpr glc_dtype v = GLC_U32; };
}  // namespace glc_detail

template <typename T>
class LeCoGPU {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "G-LeCo columns hold 32- or 64-bit integers");
  glc_ctx* ctx_ = nullptr;
  static constexpr glc_dtype kCode = glc_detail::Code<T>::v;
  static constexpr int kTileSize = 4096;  // core/CudaUtils.cuh:18 TILE_SIZE

  bool ok(glc_status s, const char* what) const {
    if (s == GLC_OK) return true;
    std::cerr << "Error: " << what << ": " << glc_status_string(s) << " (" << glc_last_error(ctx_) << ")" << std::endl;
    return false;
  }

  CompressedData<T>* wrap(glc_column* col) {
    CompressedData<T>* cd = new CompressedData<T>();
    glc_column_info info;
    glc_column_get_info(col, &info);
    cd->d_start_indices = const_cast<int32_t*>(info.d_start_indices);
    cd->d_end_indices = const_cast<int32_t*>(info.d_end_indices);
    cd->d_model_types = const_cast<int32_t*>(info.d_model_types);
    cd->d_model_params = const_cast<double*>(info.d_model_params);
    cd->d_delta_bits = const_cast<int32_t*>(info.d_delta_bits);
    cd->d_delta_array_bit_offsets = const_cast<int64_t*>(info.d_delta_array_bit_offsets);
    cd->d_error_bounds = reinterpret_cast<long long*>(const_cast<int64_t*>(info.d_error_bounds));
    cd->delta_array = const_cast<uint32_t*>(info.delta_array);
    cd->d_plain_deltas = reinterpret_cast<long long*>(const_cast<int64_t*>(info.d_plain_deltas));
    cd->num_partitions = (int)info.num_partitions;
    cd->total_values = (int)info.total_values;
    cd->d_self = cd;  // non-null like the reference's; kernels here never dereference it
    cd->glc_col = col;
    return cd;
  }

  void refresh(CompressedData<T>* cd) {
    glc_column_info info;
    glc_column_get_info(cd->glc_col, &info);
    cd->delta_array = const_cast<uint32_t*>(info.delta_array);
    cd->d_plain_deltas = reinterpret_cast<long long*>(const_cast<int64_t*>(info.d_plain_deltas));
  }

  void full(CompressedData<T>* cd, std::vector<T>& out, glc_source src) {
    if (!cd || !cd->glc_col || cd->total_values == 0) { out.clear(); return; }
    out.resize(cd->total_values);
    if (!ok(glc_decompress_full(ctx_, cd->glc_col, src, out.data(), GLC_HOST_OUT, nullptr), "decompress")) out.clear();
  }

  void ra(CompressedData<T>* cd, const std::vector<int>& pos, std::vector<T>& out, glc_source src, int fixed) {
    if (!cd || !cd->glc_col || pos.empty()) { out.clear(); return; }
    out.resize(pos.size());
    if (!ok(glc_random_access(ctx_, cd->glc_col, src, pos.data(), (int64_t)pos.size(), out.data(),
                              GLC_HOST_IN | GLC_HOST_OUT, fixed, nullptr), "random access"))
      out.clear();
  }

 public:
  LeCoGPU() {  // api/G-LeCo.cuh:103-107
    if (glc_create(&ctx_, -1) != GLC_OK) {
      std::cerr << "Error: no usable CUDA device for LeCoGPU" << std::endl;
      ctx_ = nullptr;
    }
  }
  ~LeCoGPU() {
    if (ctx_) glc_destroy(ctx_);
  }
  LeCoGPU(const LeCoGPU&) = delete;
  LeCoGPU& operator=(const LeCoGPU&) = delete;

  // api/G-LeCo.cuh:349-614.  Every partitioning runs on the GPU: variable partitioning uses the
  // split/merge partitioner (the reference's CPU partitioner's model), or, with
  // use_gpu_partitioning, the reference's GPU partitioner's boundaries (GLC_PART_VARIABLE_V6).
  // dataset_name is accepted for signature parity (no side file is written).
  CompressedData<T>* compress(const std::vector<T>& host_data_vec, bool use_variable_partitioning,
                              long long* compressed_size_bytes_result, bool use_gpu_partitioning = false,
                              const std::string& dataset_name = "") {
    (void)dataset_name;
    if (!ctx_) return nullptr;
    glc_column* col = nullptr;
    int64_t size = 0;
    const glc_partitioning mode = !use_variable_partitioning ? GLC_PART_FIXED
                                  : (use_gpu_partitioning ? GLC_PART_VARIABLE_V6 : GLC_PART_VARIABLE);
    glc_status s = glc_compress(ctx_, kCode, host_data_vec.data(), (int64_t)host_data_vec.size(), GLC_HOST_IN,
                                mode, kTileSize, &col, &size, nullptr);
    if (!ok(s, "compress")) {
      if (compressed_size_bytes_result) *compressed_size_bytes_result = 0;
      return nullptr;
    }
    if (compressed_size_bytes_result) *compressed_size_bytes_result = size;
    return wrap(col);
  }

  // api/G-LeCo.cuh:615-678
  void decompress(CompressedData<T>* cd, const std::vector<int>& positions, std::vector<T>& out) {
    ra(cd, positions, out, GLC_SRC_AUTO, 0);
  }
  // api/G-LeCo.cuh:680-693 and the variants of :166, :220, :271, :768, :1739, :1790, :1842
  void decompressFullFile(CompressedData<T>* cd, std::vector<T>& out) { full(cd, out, GLC_SRC_AUTO); }
  void decompressFullFile_BitPacked(CompressedData<T>* cd, std::vector<T>& out) { full(cd, out, GLC_SRC_PACKED); }
  void decompressFullFile_PreUnpacked(CompressedData<T>* cd, std::vector<T>& out) {
    full(cd, out, GLC_SRC_PREUNPACKED);
  }
  void decompressFullFile_OnTheFly_Optimized_V2(CompressedData<T>* cd, std::vector<T>& out) { full(cd, out, GLC_SRC_AUTO); }
  void decompressFullFile_WorkStealing(CompressedData<T>* cd, std::vector<T>& out) { full(cd, out, GLC_SRC_AUTO); }
  void decompressFullFile_WorkStealingAdvanced(CompressedData<T>* cd, std::vector<T>& out) { full(cd, out, GLC_SRC_AUTO); }
  void decompressFullFileCooperative(CompressedData<T>* cd, std::vector<T>& out) {
    if (!cd || !cd->d_plain_deltas) { out.clear(); return; }  // api/G-LeCo.cuh:284-290
    full(cd, out, GLC_SRC_PREUNPACKED);
  }
  void decompressFullFile_Fix(CompressedData<T>* cd, std::vector<T>& out, int partition_size) {
    glc_column_info info;
    if (!cd || !cd->glc_col || glc_column_get_info(cd->glc_col, &info) != GLC_OK ||
        (info.fixed_partition_len != partition_size &&
         !(info.num_partitions == 1 && info.total_values <= partition_size))) {  // one short partition
      out.clear();
      return;
    }
    full(cd, out, GLC_SRC_AUTO);
  }
  // api/G-LeCo.cuh:696-766, :1878-1928, :1931-1996
  void randomAccessPreUnpacked(CompressedData<T>* cd, const std::vector<int>& pos, std::vector<T>& out) {
    if (!cd || !cd->d_plain_deltas) { out.clear(); return; }
    ra(cd, pos, out, GLC_SRC_PREUNPACKED, 0);
  }
  void randomAccessFixed(CompressedData<T>* cd, const std::vector<int>& pos, std::vector<T>& out,
                         int fixed_partition_size) {
    if (fixed_partition_size <= 0) { out.clear(); return; }
    ra(cd, pos, out, GLC_SRC_AUTO, fixed_partition_size);
  }
  void randomAccessFixedPreUnpacked(CompressedData<T>* cd, const std::vector<int>& pos, std::vector<T>& out,
                                    int fixed_partition_size) {
    if (!cd || !cd->d_plain_deltas || fixed_partition_size <= 0) { out.clear(); return; }
    ra(cd, pos, out, GLC_SRC_PREUNPACKED, fixed_partition_size);
  }

  // api/G-LeCo.cuh:793-821
  void cleanup(CompressedData<T>* cd) {
    if (!cd) return;
    if (cd->glc_col) glc_column_free(cd->glc_col);
    delete cd;
  }

  // api/G-LeCo.cuh:826-1016 and :1999-2152 (same bytes)
  SerializedData* serialize(CompressedData<T>* cd) {
    if (!cd || !cd->glc_col) { std::cerr << "Error: Null data to serialize." << std::endl; return nullptr; }
    uint64_t size = 0;
    if (!ok(glc_blob_size(cd->glc_col, &size), "serialize")) return nullptr;
    SerializedData* sd = new SerializedData();
    sd->data = new (std::nothrow) uint8_t[size];
    if (!sd->data) { delete sd; return nullptr; }
    sd->size = size;
    uint64_t written = 0;
    if (!ok(glc_serialize(ctx_, cd->glc_col, sd->data, size, GLC_HOST_OUT, 0, &written, nullptr), "serialize")) {
      delete sd;
      return nullptr;
    }
    return sd;
  }
  SerializedData* serializeGPU(CompressedData<T>* cd) { return serialize(cd); }

  // api/G-LeCo.cuh:1019-1154 and :2157-2302: nullptr for a rejected blob
  CompressedData<T>* deserialize(const SerializedData* sd) { return deserializeGPU(sd, false); }
  CompressedData<T>* deserializeGPU(const SerializedData* sd, bool preUnpackDeltas = false) {
    if (!ctx_ || !sd || !sd->data) return nullptr;
    glc_column* col = nullptr;
    glc_status s = glc_deserialize(ctx_, kCode, sd->data, sd->size, GLC_HOST_IN, 0, preUnpackDeltas ? 1 : 0, &col,
                                   nullptr);
    if (s != GLC_OK) return nullptr;
    return wrap(col);
  }

  // api/G-LeCo.cuh:1157-1255
  DirectAccessHandle<T>* createDirectAccessHandle(const uint8_t* blob, size_t blob_size, bool copy_to_device_flag = true) {
    (void)copy_to_device_flag;  // the lookups run on the device, so the blob is always copied there
    if (!ctx_ || !blob) return nullptr;
    glc_column* col = nullptr;
    // the device copy of the blob is read in place (no deserialize), as directRandomAccessGPU does
    if (glc_attach_blob(ctx_, kCode, blob, blob_size, GLC_HOST_IN, 0, &col, nullptr) != GLC_OK) return nullptr;
    DirectAccessHandle<T>* h = new DirectAccessHandle<T>();
    h->data_blob_host = blob;
    h->data_blob_size = blob_size;
    h->glc_col = col;
    return h;
  }
  // api/G-LeCo.cuh:1257-1334
  void directRandomAccessGPU(DirectAccessHandle<T>* h, const std::vector<int>& pos, std::vector<T>& out) {
    if (!h || !h->glc_col || pos.empty()) { out.clear(); return; }
    out.resize(pos.size());
    if (!ok(glc_random_access(ctx_, h->glc_col, GLC_SRC_AUTO, pos.data(), (int64_t)pos.size(), out.data(),
                              GLC_HOST_IN | GLC_HOST_OUT, 0, nullptr), "direct random access"))
      out.clear();
  }
  // api/G-LeCo.cuh:1337-1672.  The lookups run on the device here too (this library has no
  // host decoder); the results are the same values.
  void directRandomAccessCPU(DirectAccessHandle<T>* h, const std::vector<int>& pos, std::vector<T>& out,
                             bool debug_print_flag = false) {
    (void)debug_print_flag;
    directRandomAccessGPU(h, pos, out);
  }
  // api/G-LeCo.cuh:1674-1681
  void destroyDirectAccessHandle(DirectAccessHandle<T>* h) {
    if (!h) return;
    if (h->glc_col) glc_column_free(h->glc_col);
    delete h;
  }

  // api/G-LeCo.cuh:1683-1733
  bool saveToFile(const uint8_t* data, size_t size, const std::string& filename) {
    if (!data || size == 0) return false;
    std::ofstream f(filename, std::ios::binary);
    if (!f.is_open()) return false;
    f.write(reinterpret_cast<const char*>(data), (std::streamsize)size);
    return f.good();
  }
  uint8_t* loadFromFile(const std::string& filename, size_t& size) {
    std::ifstream f(filename, std::ios::binary | std::ios::ate);
    size = 0;
    if (!f.is_open()) return nullptr;
    std::streampos end = f.tellg();
    if (end <= 0) return nullptr;
    size = (size_t)end;
    f.seekg(0, std::ios::beg);
    uint8_t* buf = new (std::nothrow) uint8_t[size];
    if (!buf) { size = 0; return nullptr; }
    f.read(reinterpret_cast<char*>(buf), (std::streamsize)size);
    if (!f.good() || (size_t)f.gcount() != size) { delete[] buf; size = 0; return nullptr; }
    return buf;
  }

  // Pre-unpacked residuals on an existing column (the preUnpackDeltas step of deserializeGPU).
  bool preUnpack(CompressedData<T>* cd, bool drop_packed = false) {
    if (!cd || !cd->glc_col) return false;
    bool r = ok(glc_preunpack(ctx_, cd->glc_col, drop_packed ? 1 : 0, nullptr), "pre-unpack");
    refresh(cd);
    return r;
  }
};

#endif  // GLC_LECO_HPP_
