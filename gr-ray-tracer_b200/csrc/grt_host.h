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

// The photon fields an output step can write, in the reference's order
// (available_output_variables, src/output/output_variables.hpp:12-18).
constexpr int kOutputFieldCount = 20;
extern const char* const kOutputFields[kOutputFieldCount];

// OutputSelection::parse (output_variables.hpp:27-70): field indices into
// kOutputFields in the order written (at most kMaxOutputSelection: up to 20
// distinct names, then "all" appends all 20); false with the reference's
// message on an unknown or empty selection.
constexpr int kMaxOutputSelection = 2 * kOutputFieldCount;
bool parse_output_variables(const std::string& spec, std::vector<int>& fields, std::string& err);

// Uncompressed (STORED) .npz writer.
class NpzOut {
public:
    // limit: the largest member, member offset and central directory a
    // non-ZIP64 archive can describe (32-bit fields); smaller only in tests
    explicit NpzOut(uint64_t limit = 0xffffffffull) : limit_(limit) {}
    bool open(const std::string& path);
    bool add(const std::string& name, const std::vector<char>& payload);
    bool close();
    // why add() or close() failed ("" when they did not)
    const std::string& error() const { return error_; }

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
    uint64_t limit_;
    std::string error_;
};

}  // namespace grt
