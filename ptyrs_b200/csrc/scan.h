// Host-side data model of a scan: PyNX position preprocessing, window corners and the seeded
// mini-batches, in double precision and bit-exact with the reference (physwkim/ptyrs
// ptyrs/src/base/positions.rs:274-315, base/addr.rs:35-127, engine/batch.rs:8-38).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace ptyb {

// `Positions::pynx_preprocess` on one axis: centre, remove a shared sub-pixel offset, snap.
std::vector<double> pynx_axis(const std::vector<double>& v, double px);

// `view_corner`: round_half_even((obj − frame)/2 + shift), or -1 when the window leaves.
int64_t view_corner(int64_t obj, int64_t frame, double shift);

// Window corners (oy, ox) per frame of preprocessed positions; false with a message when a
// window leaves the object.
bool corners_of(const std::vector<double>& y, const std::vector<double>& x, const double pixel[2],
                int ny, int nx, int nyo, int nxo, std::vector<int32_t>* out, std::string* err);

// `random_batches`: the frames 0..nframe of `epoch` as SplitMix64 Fisher–Yates batches of
// `size`, each sorted ascending, concatenated; `sizes` gets each batch's length.
void random_batches(int nframe, int size, uint64_t seed, uint64_t epoch, std::vector<int32_t>* order,
                    std::vector<int32_t>* sizes);

}  // namespace ptyb
