/* No-op stand-in for the pngwriter class so that the reference's
 * src/RPGraphLayout.cpp compiles without libpng.  PNG output is not on the
 * ForceAtlas2 path that the oracle and the CPU baseline exercise. */
#pragma once
class pngwriter {
  public:
    pngwriter(int, int, int, const char *) {}
    void invert() {}
    void filledcircle_blend(int, int, int, double, int, int, int) {}
    void line_blend(int, int, int, int, double, int, int, int) {}
    void write_png() {}
};
