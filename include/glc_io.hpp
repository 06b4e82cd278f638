// glc_io.hpp -- dataset readers of the reference's benchmark driver, for callers that load
// columns from files before compressing them (app/BenchmarkUtils.cuh:26-104), plus the SOSD
// binary format (a uint64 element count, then the values) that the reference's datasets use
// (data/download_data.sh).  Header-only host code; nothing here touches the GPU.
//
// Same names and results as the reference's readers: read_text_file parses one integer per line
// (surrounding whitespace ignored, blank lines skipped, unparsable lines skipped) and
// read_binary_file reads a raw little-endian array of T (its size must be a multiple of
// sizeof(T)).  Both return false when the file cannot be opened or read; neither prints.
#pragma once
#include <cstdint>
#include <fstream>
#include <string>
#include <type_traits>
#include <vector>

template <typename T>
bool read_text_file(const std::string& in_filename, std::vector<T>& out_data_vec) {
  static_assert(std::is_integral<T>::value, "integer columns only");
  std::ifstream f(in_filename);
  if (!f.is_open()) return false;
  out_data_vec.clear();
  std::string line;
  while (std::getline(f, line)) {
    const size_t a = line.find_first_not_of(" \t\n\r\f\v");
    if (a == std::string::npos) continue;
    const size_t b = line.find_last_not_of(" \t\n\r\f\v");
    const std::string tok = line.substr(a, b - a + 1);
    try {
      size_t used = 0;
      if (std::is_signed<T>::value) {
        const long long v = std::stoll(tok, &used);
        out_data_vec.push_back(static_cast<T>(v));
      } else {
        const unsigned long long v = std::stoull(tok, &used);
        out_data_vec.push_back(static_cast<T>(v));
      }
    } catch (const std::exception&) {
      // the reference warns and skips the line
    }
  }
  return true;
}

template <typename T>
bool read_binary_file(const std::string& in_filename, std::vector<T>& out_data_vec) {
  std::ifstream f(in_filename, std::ios::binary | std::ios::ate);
  if (!f.is_open()) return false;
  const std::streampos size = f.tellg();
  if (size < 0 || (size_t)size % sizeof(T) != 0) return false;
  out_data_vec.assign((size_t)size / sizeof(T), T());
  if (size == 0) return true;
  f.seekg(0, std::ios::beg);
  f.read(reinterpret_cast<char*>(out_data_vec.data()), (std::streamsize)size);
  if (!f.good() || (size_t)f.gcount() != (size_t)size) {
    out_data_vec.clear();
    return false;
  }
  return true;
}

// SOSD layout: uint64 count, then count values of T.
template <typename T>
bool read_sosd_file(const std::string& in_filename, std::vector<T>& out_data_vec) {
  std::ifstream f(in_filename, std::ios::binary | std::ios::ate);
  if (!f.is_open()) return false;
  const std::streampos size = f.tellg();
  if (size < 8) return false;
  f.seekg(0, std::ios::beg);
  uint64_t count = 0;
  f.read(reinterpret_cast<char*>(&count), 8);
  if (!f.good() || count > ((uint64_t)size - 8) / sizeof(T) || (uint64_t)size - 8 != count * sizeof(T)) return false;
  out_data_vec.assign((size_t)count, T());
  if (count) f.read(reinterpret_cast<char*>(out_data_vec.data()), (std::streamsize)(count * sizeof(T)));
  if (count && (!f.good() || (size_t)f.gcount() != count * sizeof(T))) {
    out_data_vec.clear();
    return false;
  }
  return true;
}
