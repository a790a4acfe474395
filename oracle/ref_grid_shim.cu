// ref_grid_shim.cu -- C entry points around the reference's own grid helpers, compiled
// from the reference sources (src/optixNSearch/grid.cu is included as it lies there).
// TEST INFRASTRUCTURE ONLY: pins the oracle's box counts and Morton ordering.
#include <vector>
#include "grid.cu"

extern "C" {

// calcSearchSize (grid.cu:84-211) on a raster count grid laid out as the reference's
// raster order, (x * dimY + y) * dimZ + z; returns the cell's mask (iteration count).
int ref_calc_search_size(int cx, int cy, int cz, unsigned dimx, unsigned dimy, unsigned dimz,
                         const unsigned* counts, float cell_size, float max_width,
                         unsigned knn) {
  GridInfo gi{};
  gi.GridDimension = make_uint3(dimx, dimy, dimz);
  std::vector<int> mask((size_t)dimx * dimy * dimz, -1);
  calcSearchSize(make_int3(cx, cy, cz), gi, false, const_cast<unsigned*>(counts), cell_size,
                 max_width, knn, mask.data());
  return mask[((size_t)cx * dimy + cy) * dimz + cz];
}

// MortonCode3 (helper_mortonCode.h:30-33).
unsigned ref_morton3(unsigned x, unsigned y, unsigned z) { return MortonCode3(x, y, z); }

// getWidthFromIter (grid.cu:33-44).
float ref_width_from_iter(int iter, float cell_size) { return getWidthFromIter(iter, cell_size); }

}
