// visa/visa.hpp -- declarations of the VISA library (davidkleiven/VISA) that
// the reference's solver sources name: the low-pass filter used for
// transverse downsampling ratios above 1 (src/solver2D.cpp:34-39, 181-185)
// and the SFML plot windows of the real-time views.  TEST INFRASTRUCTURE
// ONLY (reference pin build): the pin runs downsampling ratio 1 and no
// views, where none of this is reached; the filter throws if it ever is.
#ifndef PXP_REFSHIM_VISA_HPP
#define PXP_REFSHIM_VISA_HPP
#include <armadillo>  // the real visa.hpp brings Armadillo in
#include <stdexcept>
#include <string>

namespace visa {
enum class ArmaMatrix_t { ROW, COL, VECTOR };
template <class T, ArmaMatrix_t dim> struct ArmaGetter {
  unsigned int fixedIndx{0};
};

class GaussianKernel {};

class LowPassFilter {
 public:
  void setSourceSize(unsigned) {}
  void setTargetSize(unsigned) {}
  template <class K> void computeFilterCoefficients(const K &) {}
  template <class A, class G> void filterArray(A &, G &) {
    throw std::runtime_error("the VISA low-pass filter is not part of the reference pin build");
  }
};

struct Colormaps {
  enum class Colormap_t { VIRIDIS, GREYSCALE, NIPY_SPECTRAL };
};

class Plot {
 public:
  void setCmap(Colormaps::Colormap_t) {}
  void setOpacity(double) {}
  void setColorLim(double, double) {}
  template <class M> void setImg(const M &) {}
  template <class M> void fillVertexArray(const M &) {}
};

class WindowHandler {
 public:
  Plot &get(const std::string &) { return plot_; }
  void addPlot(const std::string &) {}
  void setLayout(unsigned, unsigned) {}
  void useSeparateDrawing() {}
  void draw() {}
  void show() {}
  void saveImg(const char *) {}

 private:
  Plot plot_;
};
}  // namespace visa
#endif
