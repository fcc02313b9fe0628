// Internal host helpers of the library: NumPy .npy reader and .npz writer.
#pragma once

#include <cstddef>
#include <cstdint>
#include <fstream>
#include <string>
#include <vector>

namespace grt {

bool npy_load_f64(const std::string& path, std::vector<size_t>& shape, std::vector<double>& data,
                  std::string& err);

// NPY 1.0 member bytes for `descr` ("<f8", "<u8", ...).
std::vector<char> npy_bytes(const char* descr, const std::vector<size_t>& shape, const void* data,
                            size_t item_size);

// Uncompressed (STORED) .npz writer.
class NpzOut {
public:
    bool open(const std::string& path);
    bool add(const std::string& name, const std::vector<char>& payload);
    bool close();

private:
    struct Entry {
        std::string name;
        uint32_t crc;
        uint32_t size;
        uint32_t offset;
    };
    std::ofstream out_;
    std::vector<Entry> entries_;
    uint64_t offset_ = 0;
};

}  // namespace grt
