// CHECKER ONLY: minimal stand-ins for the OpenCV types that HPM.h / main.h of the
// reference declare members and parameters with.  They let the reference's own
// HPM.cu (device kernels + HPM::RunPatchMatch) compile without OpenCV; none of
// the compiled reference code calls an OpenCV function.
#pragma once
#include <cstddef>
#include <vector>
namespace cv {
struct Point { int x = 0, y = 0; Point() {} Point(int a, int b) : x(a), y(b) {} };
struct Point2f { float x = 0, y = 0; };
struct Size { int width = 0, height = 0; Size() {} Size(int w, int h) : width(w), height(h) {} };
struct Rect { int x = 0, y = 0, width = 0, height = 0; };
template <class T, int N> struct Vec { T v[N]; T& operator[](int i) { return v[i]; } const T& operator[](int i) const { return v[i]; } };
typedef Vec<float, 3> Vec3f;
typedef Vec<unsigned char, 3> Vec3b;
typedef Vec<float, 6> Vec6f;
class Mat { public: int rows = 0, cols = 0; unsigned char* data = nullptr; };
template <class T> class Mat_ : public Mat {};
}  // namespace cv
