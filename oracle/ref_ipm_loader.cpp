// ORACLE — test infrastructure only (never linked into the product).
//
// A project-written definition of the reference's free function
//   bool load_interaction_potential_offline_sample_set_file(
//       const std::filesystem::path&, InteractionPotentialOfflineSampleSet&, std::string*)
// (declared at src/core/physics/collisions/InteractionPotentialOfflineSampleSet.h:100-104).
// The reference reads HDF5 there; HDF5 is absent from this image, so this
// definition reads the same fields from a flat little-endian file written by
// tests/golden/make_ipm_golden.py.  Linked into oracle/_ref/ref_harness next
// to the reference's own InteractionPotentialCollisionHandler.cpp, it lets
// the reference's runtime sampler (handle_collision,
// InteractionPotentialCollisionHandler.cpp:298-552) run unchanged.
//
// File layout:
//   char[8]  "ICBIPMS1"
//   int64    n_orient, n_bins, n_samples, gas_len
//   char     gas[gas_len]
//   double   logv_bins[n_bins]
//   double   sigma_mt_m2[n_orient * n_bins], sigma_event_m2[...], b_max_m[...]
//   int64    cdf_offsets[n_orient * n_bins], cdf_counts[...]
//   double   cdf_values[n_samples], dp_samples[3 * n_samples]
//   double   dp_stats[4 * n_orient * n_bins]
#include "core/physics/collisions/InteractionPotentialOfflineSampleSet.h"

#include <cstdint>
#include <cstdio>
#include <cstring>

namespace ICARION::physics {

namespace {

template <class T>
bool read_array(FILE* f, std::vector<T>& v, size_t n) {
    v.resize(n);
    return n == 0 || std::fread(v.data(), sizeof(T), n, f) == n;
}

bool fail(std::string* err, const std::string& msg) {
    if (err) *err = msg;
    return false;
}

}  // namespace

bool load_interaction_potential_offline_sample_set_file(const std::filesystem::path& path,
                                                        InteractionPotentialOfflineSampleSet& out,
                                                        std::string* error_msg) {
    FILE* f = std::fopen(path.string().c_str(), "rb");
    if (!f) return fail(error_msg, "cannot open " + path.string());
    struct Closer {
        FILE* f;
        ~Closer() { std::fclose(f); }
    } closer{f};
    char magic[8];
    int64_t hdr[4];
    if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, "ICBIPMS1", 8) != 0)
        return fail(error_msg, "not a sample-set file: " + path.string());
    if (std::fread(hdr, sizeof(int64_t), 4, f) != 4) return fail(error_msg, "short header");
    const int64_t n_orient = hdr[0], n_bins = hdr[1], n_samples = hdr[2], gas_len = hdr[3];
    if (n_orient <= 0 || n_bins <= 0 || n_samples < 0 || gas_len < 0 || gas_len > 256)
        return fail(error_msg, "bad header");
    out = InteractionPotentialOfflineSampleSet{};
    out.gas.resize(static_cast<size_t>(gas_len));
    if (gas_len > 0 && std::fread(out.gas.data(), 1, static_cast<size_t>(gas_len), f) != static_cast<size_t>(gas_len))
        return fail(error_msg, "short gas name");
    out.n_orient = static_cast<size_t>(n_orient);
    out.n_bins = static_cast<size_t>(n_bins);
    const size_t cells = out.n_orient * out.n_bins;
    const size_t ns = static_cast<size_t>(n_samples);
    const bool ok = read_array(f, out.logv_bins, out.n_bins) && read_array(f, out.sigma_mt_m2, cells) &&
                    read_array(f, out.sigma_event_m2, cells) && read_array(f, out.b_max_m, cells) &&
                    read_array(f, out.cdf_offsets, cells) && read_array(f, out.cdf_counts, cells) &&
                    read_array(f, out.cdf_values, ns) && read_array(f, out.dp_samples, 3 * ns) &&
                    read_array(f, out.dp_stats, 4 * cells);
    if (!ok) return fail(error_msg, "short sample-set file " + path.string());
    return true;
}

}  // namespace ICARION::physics
