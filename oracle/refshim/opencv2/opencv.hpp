// opencv2/opencv.hpp -- HOST STAND-IN (TEST INFRASTRUCTURE: the reference-pinned oracle under
// oracle/_ref).  The reference's DPE.h / main.h include OpenCV for cv::Mat and a few image
// functions; the OpenCV C++ library is not installed here.  This header declares the part of the
// public OpenCV API that DPE.cu and DPE.cpp name, with OpenCV's documented meanings:
//   * cv::Mat: rows x cols of one element type (CV_8U/8S/16U/16S/32S/32F/64F, 1-4 channels,
//     type = depth + 8 * (channels - 1)), continuous, shared on copy, deep-copied by clone();
//   * cv::Vec / Size / Point / Scalar as small value types;
//   * MIN / MAX as OpenCV's macros (cvdef.h): ((a) > (b) ? (b) : (a)) and ((a) < (b) ? (b) : (a)).
// imread decodes binary PGM / PPM (P5 / P6) files whatever their extension (the harness writes
// the test images that way: gray as PGM, colour as PPM, returned in BGR order as OpenCV does).  Functions of the
// reference that the per-view PatchMatch and fusion paths never call (Canny, HoughLinesP, resize
// between different sizes, threshold, line, imwrite) exist only so the files link, and stop the
// process with a message if called.
#ifndef REFSHIM_OPENCV_HPP_
#define REFSHIM_OPENCV_HPP_

#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

typedef unsigned char uchar;
typedef unsigned short ushort;
typedef signed char schar;

#define CV_8U 0
#define CV_8S 1
#define CV_16U 2
#define CV_16S 3
#define CV_32S 4
#define CV_32F 5
#define CV_64F 6
#define CV_MAKETYPE(depth, cn) ((depth) + (((cn) - 1) << 3))
#define CV_8UC1 CV_MAKETYPE(CV_8U, 1)
#define CV_8UC3 CV_MAKETYPE(CV_8U, 3)
#define CV_32SC1 CV_MAKETYPE(CV_32S, 1)
#define CV_32FC1 CV_MAKETYPE(CV_32F, 1)
#define CV_32FC3 CV_MAKETYPE(CV_32F, 3)
#define CV_32FC4 CV_MAKETYPE(CV_32F, 4)
#define CV_PI 3.1415926535897932384626433832795
#ifndef MIN
#define MIN(a, b) ((a) > (b) ? (b) : (a))
#endif
#ifndef MAX
#define MAX(a, b) ((a) < (b) ? (b) : (a))
#endif

namespace cv {

enum { IMREAD_GRAYSCALE = 0, IMREAD_COLOR = 1 };
enum { INTER_NEAREST = 0, INTER_LINEAR = 1 };
enum { THRESH_BINARY = 0 };

template <class T, int n> struct Vec {
  T val[n];
  Vec() { for (int i = 0; i < n; ++i) val[i] = T(0); }
  Vec(T a, T b, T c) : Vec() { val[0] = a; if (n > 1) val[1] = b; if (n > 2) val[2] = c; }
  Vec(T a, T b, T c, T d) : Vec() { val[0] = a; val[1] = b; val[2] = c; if (n > 3) val[3] = d; }
  T &operator[](int i) { return val[i]; }
  const T &operator[](int i) const { return val[i]; }
};
template <class T, int n, class S> Vec<T, n> operator/(const Vec<T, n> &v, S s) {
  Vec<T, n> r;
  for (int i = 0; i < n; ++i) r.val[i] = (T)(v.val[i] / s);
  return r;
}
template <class T, int n, class S> Vec<T, n> operator*(const Vec<T, n> &v, S s) {
  Vec<T, n> r;
  for (int i = 0; i < n; ++i) r.val[i] = (T)(v.val[i] * s);
  return r;
}
typedef Vec<float, 3> Vec3f;
typedef Vec<uchar, 3> Vec3b;
typedef Vec<int, 4> Vec4i;
typedef Vec<float, 4> Vec4f;

template <class T> struct Size_ {
  T width = 0, height = 0;
  Size_() = default;
  Size_(T w, T h) : width(w), height(h) {}
  bool operator==(const Size_ &o) const { return width == o.width && height == o.height; }
  bool operator!=(const Size_ &o) const { return !(*this == o); }
};
typedef Size_<int> Size2i;
typedef Size2i Size;

struct Point {
  int x = 0, y = 0;
  Point() = default;
  Point(int a, int b) : x(a), y(b) {}
};

struct Scalar {
  double val[4] = {0, 0, 0, 0};
  Scalar() = default;
  Scalar(double a, double b = 0, double c = 0, double d = 0) { val[0] = a; val[1] = b; val[2] = c; val[3] = d; }
};

int ref_depth_bytes(int depth);

class Mat {
 public:
  struct MatStep {
    size_t p[2] = {0, 0};
    size_t operator[](int i) const { return p[i]; }
    operator size_t() const { return p[0]; }
  };
  int rows = 0, cols = 0;
  uchar *data = nullptr;
  MatStep step;

  Mat() = default;
  Mat(int r, int c, int type) { create(r, c, type); }
  Mat(int r, int c, int type, const Scalar &s) { create(r, c, type); setTo(s); }
  Mat(Size sz, int type) { create(sz.height, sz.width, type); }
  Mat(Size sz, int type, const Scalar &s) { create(sz.height, sz.width, type); setTo(s); }

  void create(int r, int c, int type);
  void setTo(const Scalar &s);
  int type() const { return type_; }
  int depth() const { return type_ & 7; }
  int channels() const { return (type_ >> 3) + 1; }
  size_t elemSize() const { return (size_t)ref_depth_bytes(depth()) * channels(); }
  size_t total() const { return (size_t)rows * cols; }
  bool empty() const { return data == nullptr || total() == 0; }
  Size size() const { return Size(cols, rows); }
  Mat clone() const;
  void convertTo(Mat &dst, int rtype, double alpha = 1.0, double beta = 0.0) const;
  template <class T> T *ptr(int r = 0) { return reinterpret_cast<T *>(data + (size_t)r * step.p[0]); }
  template <class T> const T *ptr(int r = 0) const { return reinterpret_cast<const T *>(data + (size_t)r * step.p[0]); }
  template <class T> T &at(int r, int c) { return ptr<T>(r)[c]; }
  template <class T> const T &at(int r, int c) const { return ptr<T>(r)[c]; }
  static Mat zeros(int r, int c, int type) { return Mat(r, c, type, Scalar(0)); }
  static Mat zeros(Size sz, int type) { return Mat(sz.height, sz.width, type, Scalar(0)); }

 private:
  int type_ = 0;
  std::shared_ptr<std::vector<uchar>> buf_;
};

Mat imread(const std::string &filename, int flags = IMREAD_COLOR);
bool imwrite(const std::string &filename, const Mat &img, const std::vector<int> &params = std::vector<int>());
void resize(const Mat &src, Mat &dst, Size dsize, double fx = 0, double fy = 0, int interpolation = INTER_LINEAR);
double threshold(const Mat &src, Mat &dst, double thresh, double maxval, int type);
void Canny(const Mat &image, Mat &edges, double threshold1, double threshold2, int aperture_size = 3,
           bool l2_gradient = false);
void HoughLinesP(const Mat &image, std::vector<Vec4i> &lines, double rho, double theta, int threshold,
                 double min_line_length = 0, double max_line_gap = 0);
void line(Mat &img, Point a, Point b, const Scalar &color, int thickness = 1);

}  // namespace cv

#endif
