// pointio.h -- point-cloud files for the optixNSearch CLI.
#pragma once
#include <cstddef>
#include <string>
#include <vector>

namespace rtnn {

// Reads the points of `path` as x,y,z float triples.
//   *.bin / *.f32: raw little-endian float32 x,y,z triples (size a multiple of 12 bytes).
//   anything else: text, one "x,y,z" point per line, each field read as a correctly rounded
//   double and cast to float -- the values the reference's reader gives
//   (src/optixNSearch/util.cpp:101-135, sscanf "%lf,%lf,%lf"). A line whose fields do not
//   all parse keeps 0 for the fields that did not (the reference leaves them unset).
// Text is parsed on `threads` host threads (0: all hardware threads). Returns false and
// fills `err` when the file cannot be read or a binary file has a ragged size.
bool read_points_file(const std::string& path, unsigned threads, std::vector<float>* xyz,
                      std::string* err);

// Writes x,y,z float triples as a raw little-endian float32 file.
bool write_points_f32(const std::string& path, const std::vector<float>& xyz, std::string* err);

// True for the names read as raw float32 (*.bin, *.f32).
bool is_binary_points_name(const std::string& path);

}  // namespace rtnn
