// File helpers shared by the drop-in executables: the u32 matrix files
// ("u32 dim[2]" + dim[0] x dim[1] u32, little-endian), raw float64 weight
// files, device choice, and the reference tools' stdout conventions.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace tool {

// Reads a matrix file; returns false if it cannot be opened.  Missing body
// values (short file) are left zero, like the reference's unchecked fread.
bool read_mat(const std::string& path, uint32_t& d0, uint32_t& d1, std::vector<uint32_t>& data);
bool read_header(const std::string& path, uint32_t& d0, uint32_t& d1);
bool read_f64(const std::string& path, size_t n, std::vector<double>& out);
bool write_mat(const std::string& path, uint32_t d0, uint32_t d1, const uint32_t* data, size_t n);
bool write_raw(const std::string& path, const void* data, size_t bytes, bool append = false);

// Picks the GPU like the reference tools do (random device per process,
// cu/joinEdgeIndel.cu:248-252); CASPHY_DEVICE overrides.  Returns the index.
int pick_device();
double now_s();
int fail(const char* tool, int status);

}  // namespace tool
