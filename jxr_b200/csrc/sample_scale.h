// sample_scale.h -- the scale of reduced-resolution samples.
//
// A quarter-resolution decode stops after the first level: one sample a
// block, the block's DC coefficient.  A sixteenth stops before it: one sample
// a macroblock, its DC (or, with two-level overlap, the first-level picture
// of the DC band summed over the macroblock).  Neither value is at the level
// of the samples it stands for: the transforms skipped divide by a power of
// two, and under overlap filtering the filters skipped change a flat area by
// a factor that is no power of two, plus an offset the forward filters'
// rounding leaves.  The reference measures both on flat probe images run through the
// analysis and the reduced decode (SampleScale,
// crates/jxr-native/src/reconstruct/sample_scale.rs:155-350); this restates it.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace jxr {

struct QuarterScale {
    int32_t shift = -1;                 // >= 0: samples >>= shift (no overlap filtering)
    int64_t gain = 0;                   // multiplier of a coefficient (flat terms)
    uint32_t probe_stride = 0;          // samples across the probe picture
    std::vector<int64_t> divisor, bias; // per probe-picture sample
    std::vector<uint32_t> columns, rows;// per component-picture column / row: its probe column / row
};

// The scale of the reduced picture, at 1/`denominator` of the resolution (4:
// one sample a block, 16: one sample a macroblock), of a plane of `mbs_x` x
// `mbs_y` macroblocks of `bc` x `br` blocks, whose overlap regions have the
// macroblock boundaries `cols` / `rows` (0 .. extent, tile boundaries when
// hard, else the plane).  Returns false with `why` set when the probe's own
// arithmetic fails.
bool reduced_scale(int denominator, int bc, int br, bool scale2, int overlap, uint32_t mbs_x, uint32_t mbs_y,
                   const std::vector<uint32_t> &cols, const std::vector<uint32_t> &rows, QuarterScale &out,
                   std::string &why);

}  // namespace jxr
