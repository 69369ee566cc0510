// mrc.hpp -- MRC2014 image files: reading modes 0, 1, 2, 6 and 12 (as the
// reference's MRCFile does for input stacks and volumes,
// src/core/mrc_file.cpp) and writing mode 2 with the pixel size in the cell
// dimensions (Image::QuickAndDirtyWriteSlice, src/core/image.cpp:5548-5556;
// src/core/mrc_header.cpp:99-140).
#pragma once
#include <string>
#include <vector>

namespace tmhost {

struct MrcData {
    int nx = 0, ny = 0, nz = 0;
    float pixel_size = 0.f;        // cell_a_x / mx, 0 when the cell is unset
    std::vector<float> data;       // [z][y][x]
};

// Reads slices [first, last] (1-based, inclusive; last = 0 means all).
bool read_mrc(const std::string& path, MrcData& out, std::string& err, int first_slice = 1, int last_slice = 0);

// Writes an nx*ny*nz float volume (mode 2).
bool write_mrc(const std::string& path, int nx, int ny, int nz, const float* data, float pixel_size, std::string& err);

}  // namespace tmhost
