// icp_record_io.cpp -- see icp_record_io.hpp.
#include "icp_record_io.hpp"

#include <bit>
#include <charconv>
#include <cmath>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>
#include <stdexcept>

#include "icp_host_math.hpp"

namespace icp::io {

void write_npy_f64(const std::filesystem::path& path, const std::vector<uint64_t>& shape, const double* data,
                   size_t count)
{
    static_assert(std::endian::native == std::endian::little, "little-endian host required");
    if (shape.empty() || shape.size() > 8) throw std::invalid_argument("NPY: require 1..8 dimensions.");
    uint64_t n = 1;
    std::string dims = "(";
    for (const uint64_t d : shape) {
        if (d == 0 || n > std::numeric_limits<uint64_t>::max() / d) throw std::length_error("NPY: invalid shape.");
        n *= d;
        dims += std::to_string(d) + ", ";
    }
    dims += ")";
    if (n != count) throw std::logic_error("NPY: element count differs from shape.");
    std::string header = "{'descr': '<f8', 'fortran_order': False, 'shape': " + dims + ", }";
    const size_t pad = (64 - (10 + header.size() + 1) % 64) % 64;
    header.append(pad, ' ');
    header.push_back('\n');
    if (header.size() > 65535) throw std::length_error("NPY: header too large.");
    std::ofstream out(path, std::ios::binary | std::ios::trunc);
    if (!out) throw std::runtime_error("NPY: cannot open " + path.string());
    const unsigned char prefix[10] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0, (unsigned char)(header.size() & 255u),
                                      (unsigned char)(header.size() >> 8)};
    out.write(reinterpret_cast<const char*>(prefix), 10);
    out.write(header.data(), (std::streamsize)header.size());
    out.write(reinterpret_cast<const char*>(data), (std::streamsize)(count * sizeof(double)));
    out.flush();
    if (!out) throw std::runtime_error("NPY: write failed for " + path.string());
}

StagingDirectory::StagingDirectory(const std::filesystem::path& destination) : destination_(destination)
{
    const auto name = destination_.filename();
    if (destination_.empty() || name.empty() || name == "." || name == ".." || destination_.extension() == ".part")
        throw std::invalid_argument("Invalid dataset destination.");
    staging_ = destination_;
    staging_ += ".part";
    if (std::filesystem::exists(destination_)) throw std::runtime_error("Dataset already exists; refusing to overwrite.");
    if (!destination_.parent_path().empty()) std::filesystem::create_directories(destination_.parent_path());
    if (!std::filesystem::create_directory(staging_))
        throw std::runtime_error("Staging directory exists; inspect/retire the previous .part directory.");
}

void StagingDirectory::commit()
{
    if (committed_ || !std::filesystem::is_regular_file(staging_ / "metadata.json"))
        throw std::logic_error("Dataset has no complete metadata or was already committed.");
    if (std::filesystem::exists(destination_)) throw std::runtime_error("Destination appeared while writing.");
    std::filesystem::rename(staging_, destination_);
    committed_ = true;
}

namespace {

// Round constants: first 32 bits of the fractional parts of the cube roots of the first 64
// primes; initial state: of the square roots of the first 8 primes (FIPS 180-4, 4.2.2/5.3.3).
struct ShaConstants {
    uint32_t k[64], h[8];
    ShaConstants()
    {
        int found = 0;
        for (int p = 2; found < 64; ++p) {
            bool prime = true;
            for (int d = 2; d * d <= p; ++d)
                if (p % d == 0) prime = false;
            if (!prime) continue;
            const long double c = std::cbrt((long double)p);
            k[found] = (uint32_t)std::floor((c - std::floor(c)) * 4294967296.0L);
            if (found < 8) {
                const long double r = std::sqrt((long double)p);
                h[found] = (uint32_t)std::floor((r - std::floor(r)) * 4294967296.0L);
            }
            ++found;
        }
    }
};
const ShaConstants& sha_constants()
{
    static const ShaConstants c;
    return c;
}
inline uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

} // namespace

std::string sha256_hex(std::string_view data)
{
    const ShaConstants& C = sha_constants();
    uint32_t h[8];
    std::memcpy(h, C.h, sizeof h);
    std::string msg(data);
    const uint64_t bits = (uint64_t)data.size() * 8u;
    msg.push_back((char)0x80);
    while (msg.size() % 64 != 56) msg.push_back('\0');
    for (int i = 7; i >= 0; --i) msg.push_back((char)((bits >> (8 * i)) & 0xffu));
    for (size_t off = 0; off < msg.size(); off += 64) {
        uint32_t w[64];
        for (int t = 0; t < 16; ++t) {
            const auto* b = reinterpret_cast<const unsigned char*>(msg.data() + off + 4 * t);
            w[t] = (uint32_t)b[0] << 24 | (uint32_t)b[1] << 16 | (uint32_t)b[2] << 8 | (uint32_t)b[3];
        }
        for (int t = 16; t < 64; ++t) {
            const uint32_t s0 = rotr(w[t - 15], 7) ^ rotr(w[t - 15], 18) ^ (w[t - 15] >> 3);
            const uint32_t s1 = rotr(w[t - 2], 17) ^ rotr(w[t - 2], 19) ^ (w[t - 2] >> 10);
            w[t] = w[t - 16] + s0 + w[t - 7] + s1;
        }
        uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], k = h[7];
        for (int t = 0; t < 64; ++t) {
            const uint32_t t1 = k + (rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)) + ((e & f) ^ (~e & g)) + C.k[t] + w[t];
            const uint32_t t2 = (rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
            k = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
        }
        h[0] += a; h[1] += b; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += k;
    }
    static const char* hex = "0123456789abcdef";
    std::string out;
    for (const uint32_t v : h)
        for (int s = 28; s >= 0; s -= 4) out.push_back(hex[(v >> s) & 15u]);
    return out;
}

namespace {
std::string_view trim(std::string_view s)
{
    const auto a = s.find_first_not_of(" \t\r");
    if (a == std::string_view::npos) return {};
    return s.substr(a, s.find_last_not_of(" \t\r") - a + 1);
}
template <class T> T number(std::string_view s)
{
    s = trim(s);
    T v{};
    const auto r = std::from_chars(s.data(), s.data() + s.size(), v);
    if (s.empty() || r.ec != std::errc{} || r.ptr != s.data() + s.size())
        throw std::invalid_argument("Malformed orientation number.");
    return v;
}
} // namespace

Plan parse_plan(std::string_view csv)
{
    Plan plan;
    plan.sha256 = sha256_hex(csv);
    host::KahanSum weights;
    bool header = false;
    size_t start = 0, line_no = 0;
    while (start < csv.size()) {
        const size_t end = csv.find('\n', start);
        const auto line = trim(csv.substr(start, (end == std::string_view::npos ? csv.size() : end) - start));
        start = end == std::string_view::npos ? csv.size() : end + 1;
        ++line_no;
        if (line.empty() || line.front() == '#') continue;
        try {
            if (!header) {
                if (line != "qw,qx,qy,qz,weight,samples,seed")
                    throw std::invalid_argument("Expected CSV header qw,qx,qy,qz,weight,samples,seed.");
                header = true;
                continue;
            }
            std::array<std::string_view, 7> col;
            size_t pos = 0;
            for (unsigned c = 0; c < 7; ++c) {
                const size_t comma = line.find(',', pos);
                if ((c < 6 && comma == std::string_view::npos) || (c == 6 && comma != std::string_view::npos))
                    throw std::invalid_argument("Expected seven CSV fields.");
                col[c] = line.substr(pos, (comma == std::string_view::npos ? line.size() : comma) - pos);
                pos = comma + 1;
            }
            PlanNode n;
            for (unsigned c = 0; c < 4; ++c) n.q[c] = number<double>(col[c]);
            double r[9];
            if (!host::rotation(n.q[0], n.q[1], n.q[2], n.q[3], r))
                throw std::invalid_argument("Quaternion must be unit length (w,x,y,z).");
            n.weight = number<double>(col[4]);
            n.samples = number<uint64_t>(col[5]);
            n.seed = number<uint64_t>(col[6]);
            if (!host::finite(n.weight) || !(n.weight > 0) || !n.samples)
                throw std::invalid_argument("Weights and sample counts must be positive.");
            if (n.samples > std::numeric_limits<uint64_t>::max() - plan.total_samples)
                throw std::overflow_error("Planned sample count overflows.");
            plan.total_samples += n.samples;
            weights.add(n.weight);
            plan.nodes.push_back(n);
        } catch (const std::exception& e) {
            throw std::invalid_argument("Orientation CSV line " + std::to_string(line_no) + ": " + e.what());
        }
    }
    if (!header || plan.nodes.empty() || !host::finite(weights.value) || std::fabs(weights.value - 1) > 2e-12)
        throw std::invalid_argument("Orientation number-probability weights must sum to one (within 2e-12).");
    plan.input_weight_sum = weights.value;
    for (auto& n : plan.nodes) n.weight /= weights.value;
    return plan;
}

Plan read_plan(const std::filesystem::path& p)
{
    const auto bytes = std::filesystem::file_size(p);
    if (bytes > 256ull * 1024 * 1024) throw std::length_error("Orientation plan exceeds explicit 256 MiB input limit.");
    std::ifstream in(p, std::ios::binary);
    if (!in) throw std::runtime_error("Cannot read orientation plan.");
    std::string data((size_t)bytes, '\0');
    in.read(data.data(), (std::streamsize)bytes);
    if (in.gcount() != (std::streamsize)bytes) throw std::runtime_error("Short/changed orientation file.");
    return parse_plan(data);
}

std::string json_quote(std::string_view s)
{
    static const char* hex = "0123456789abcdef";
    std::string o = "\"";
    for (const unsigned char c : s) {
        if (c == '"' || c == '\\') {
            o.push_back('\\');
            o.push_back((char)c);
        } else if (c < 32) {
            o += "\\u00";
            o.push_back(hex[c >> 4]);
            o.push_back(hex[c & 15]);
        } else
            o.push_back((char)c);
    }
    o.push_back('"');
    return o;
}

} // namespace icp::io
