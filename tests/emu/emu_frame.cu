// Host check of the ghost-frame enumeration that k_copy_frame uses
// (frame_cells / frame_offset in dim2d_kernels.cuh): for several field
// shapes and pitches, the offsets of cells 0 .. frame_cells-1 hit every cell
// within BC of an edge of the 4 planes exactly once and nothing else (the
// interior and the pitch padding are never touched).
// Used by tests/test_frame_emulation.py.
#include <cstdio>
#include <vector>

#include "../../dim2d_finite_volume_b200/csrc/dim2d_kernels.cuh"

using namespace dim2d;

int main() {
  const int shapes[][3] = {{8, 8, 16},      {9, 13, 16},    {68, 52, 80},
                           {132, 132, 144}, {33, 97, 48},   {1028, 260, 1040},
                           {2052, 2052, 2064}};
  long bad = 0;
  for (const auto& s : shapes) {
    Field f;
    f.nx = s[0];
    f.ny = s[1];
    f.pitch = s[2];
    f.plane = (size_t)f.ny * f.pitch;
    std::vector<int> hits(4 * f.plane, 0);
    const int n = frame_cells(f);
    for (int i = 0; i < n; i++) {
      const size_t o = frame_offset(f, i);
      if (o >= hits.size()) {
        bad++;
        continue;
      }
      hits[o]++;
    }
    long cells = 0;
    for (int v = 0; v < 4; v++)
      for (int y = 0; y < f.ny; y++)
        for (int x = 0; x < f.pitch; x++) {
          const bool ghost =
              x < f.nx && (x < BC || x >= f.nx - BC || y < BC || y >= f.ny - BC);
          const int h = hits[(size_t)v * f.plane + (size_t)y * f.pitch + x];
          if (h != (ghost ? 1 : 0)) bad++;
          cells += ghost;
        }
    if (cells != n) bad++;
    std::printf("%d x %d, pitch %d: %d frame cells\n", f.nx, f.ny, f.pitch, n);
  }
  std::printf("bad %ld\n", bad);
  return bad ? 1 : 0;
}
