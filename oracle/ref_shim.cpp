// Test-infrastructure shim over the REFERENCE e8qlib public API.
//
// Compiled by oracle/Makefile against the reference's own sources (never
// copied into this repository) into oracle/_ref/libe8qref.so. It exists only
// so the golden-vector generator (tests/golden/make_golden.py) and the CPU
// tests can call single reference functions through ctypes; nothing in the
// product links or loads it.
//
// Every function mirrors one public reference entry point:
//   BranchLevels / FixedScale / EncodeVectorAtScale / BuildRefineTables /
//   PackRefineBlock     include/e8qlib/quantization/e8q_codec.hpp:48-146
//   PackCoarseRow       include/e8qlib/index/e8q.hpp:314-316
//   FhtKac4Rotator      include/e8qlib/utils/rotator.hpp:17-42
#include <cstdint>
#include <cstring>
#include <vector>

#include "e8qlib/index/e8q.hpp"
#include "e8qlib/quantization/e8q_codec.hpp"
#include "e8qlib/utils/rotator.hpp"

extern "C" {

int ref_branch_levels(int bits, int branch, double* out) {
    const std::vector<double> lev = e8qlib::BranchLevels(bits, branch);
    std::memcpy(out, lev.data(), lev.size() * sizeof(double));
    return static_cast<int>(lev.size());
}

double ref_fixed_scale(int bits) { return e8qlib::FixedScale(bits); }

// n unit vectors of padded_dim floats -> digits[n][B][8] (uint16), branch[n][B].
int ref_encode(const float* unit, size_t n, int padded_dim, int bits, double s,
               uint16_t* digits, uint8_t* branch) {
    const int blocks = padded_dim / 8;
    e8qlib::VectorCode vc;
    for (size_t r = 0; r < n; ++r) {
        e8qlib::EncodeVectorAtScaleInto(unit + r * static_cast<size_t>(padded_dim), padded_dim,
                                        bits, s, vc);
        for (int b = 0; b < blocks; ++b) {
            for (int i = 0; i < 8; ++i) {
                digits[(r * blocks + b) * 8 + i] = vc.digits[b][i];
            }
            branch[r * blocks + b] = static_cast<uint8_t>(vc.branch[b]);
        }
    }
    return 0;
}

size_t ref_rotator_sign_bytes(size_t dim, uint64_t seed) {
    e8qlib::FhtKac4Rotator rot(dim, seed);
    return rot.dump_bytes();
}

void ref_rotator_signs(size_t dim, uint64_t seed, uint8_t* out) {
    e8qlib::FhtKac4Rotator rot(dim, seed);
    std::vector<char> buf(rot.dump_bytes());
    rot.Save(buf.data());
    std::memcpy(out, buf.data(), buf.size());
}

// n rows of dim floats -> n rows of padded_dim floats.
void ref_rotate(size_t dim, uint64_t seed, const float* src, size_t n, float* dst) {
    e8qlib::FhtKac4Rotator rot(dim, seed);
    const size_t pd = rot.padded_dim();
    for (size_t r = 0; r < n; ++r) {
        rot.Rotate(src + r * dim, dst + r * pd);
    }
}

int ref_refine_tables(int bits, int padded_dim, float* out) {
    const std::vector<float> t = e8qlib::BuildRefineTables(bits, padded_dim);
    std::memcpy(out, t.data(), t.size() * sizeof(float));
    return static_cast<int>(t.size());
}

void ref_pack_block(const uint16_t digits[8], int branch, int bits, uint8_t* rowa,
                    uint8_t* refine) {
    e8qlib::PackCoarseRow(digits, branch, bits, 0, rowa);
    if (bits >= 2) {
        e8qlib::PackRefineBlock(digits, branch, bits, refine);
    }
}

void ref_scan_class_means(int bits, double* w_cls) { e8qlib::ScanClassMeans(bits, w_cls); }

}  // extern "C"
