// icp_record_io.hpp -- record output contract shared by the command-line drop-ins.
//
// NPY v1 files of little-endian binary64 in C order (header padded so that the data starts
// on a 64-byte boundary, the dictionary text formatted like the reference's writer so that
// files are byte-identical: src/npy_writer.cpp:18-95), the `.part` staging directory that
// is renamed into place only after metadata.json exists (src/npy_writer.cpp:97-121), the
// orientation CSV (hex_phase/src/orientation_plan.cpp:69-120) with the SHA-256 digest of its
// bytes, and JSON helpers.
#pragma once
#include <array>
#include <cstdint>
#include <filesystem>
#include <string>
#include <string_view>
#include <vector>

namespace icp::io {

// Writes one NPY v1 <f8 C-order array of the given shape (all at once).
void write_npy_f64(const std::filesystem::path& path, const std::vector<uint64_t>& shape, const double* data,
                   size_t count);

// Creates <destination>.part exclusively; commit() renames it to <destination>.
class StagingDirectory {
public:
    explicit StagingDirectory(const std::filesystem::path& destination);
    const std::filesystem::path& staging() const { return staging_; }
    void commit();

private:
    std::filesystem::path destination_, staging_;
    bool committed_ = false;
};

// FIPS 180-4 SHA-256 of a byte string, lower-case hex.
std::string sha256_hex(std::string_view bytes);

struct PlanNode {
    double q[4] = {};
    double weight = 0;
    uint64_t samples = 0, seed = 0;
};
struct Plan {
    std::vector<PlanNode> nodes;
    uint64_t total_samples = 0;
    double input_weight_sum = 0;
    std::string sha256;
};
// Parses "qw,qx,qy,qz,weight,samples,seed" rows; weights must sum to one within 2e-12 and
// are then divided by their (compensated) sum.  Throws std::invalid_argument.
Plan parse_plan(std::string_view csv);
Plan read_plan(const std::filesystem::path& path);

// JSON string literal with the control-character escapes used by the metadata writers.
std::string json_quote(std::string_view s);

} // namespace icp::io
