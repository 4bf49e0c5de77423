// CHECKER ONLY: stand-ins for the OpenCV API that the reference's host sources
// (main.cpp, HPM.cpp of HPM-MVS++) use, so that oracle/ref_host.mk can compile
// those files from their own sources and run two of their stages,
// ConfidenceEvaluation and RunFusion, on the CPU (oracle/ref_host_driver.cpp).
//
// cv::Mat keeps OpenCV's semantics where those stages rely on them: copies
// share reference-counted storage, clone() deep-copies, release() drops this
// handle, zeros() allocates zero-filled storage, rows x cols elements of a
// CV_<depth>C<channels> type, row-major and continuous.  cv::imread reads a
// raw sidecar file written by the caller (<path>.raw: int32 rows, cols,
// channels, then uint8 pixels) in place of decoding the image.  Functions that
// the two stages never reach are declared only; the linker drops their callers.
#pragma once
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

typedef unsigned char uchar;
typedef signed char schar;
typedef unsigned short ushort;

#define CV_8U 0
#define CV_8S 1
#define CV_16U 2
#define CV_16S 3
#define CV_32S 4
#define CV_32F 5
#define CV_64F 6
#define CV_CN_SHIFT 3
#define CV_MAKETYPE(depth, cn) (((depth) & 7) + (((cn) - 1) << CV_CN_SHIFT))
#define CV_8UC1 CV_MAKETYPE(CV_8U, 1)
#define CV_8UC3 CV_MAKETYPE(CV_8U, 3)
#define CV_32FC1 CV_MAKETYPE(CV_32F, 1)
#define CV_32FC2 CV_MAKETYPE(CV_32F, 2)
#define CV_32FC3 CV_MAKETYPE(CV_32F, 3)
#define CV_32SC1 CV_MAKETYPE(CV_32S, 1)
#define CV_64FC1 CV_MAKETYPE(CV_64F, 1)
#define CV_PI 3.1415926535897932384626433832795

namespace cv {

inline int depth_bytes(int type) {
    static const int b[8] = {1, 1, 2, 2, 4, 4, 8, 0};
    return b[type & 7];
}
inline int type_channels(int type) { return (type >> CV_CN_SHIFT) + 1; }

template <class T, int N>
struct Vec {
    T v[N];
    Vec() { for (int i = 0; i < N; ++i) v[i] = T(); }
    Vec(T a, T b, T c) { static_assert(N >= 3, "Vec"); v[0] = a; v[1] = b; v[2] = c; for (int i = 3; i < N; ++i) v[i] = T(); }
    T& operator[](int i) { return v[i]; }
    const T& operator[](int i) const { return v[i]; }
    T& operator()(int i) { return v[i]; }
    const T& operator()(int i) const { return v[i]; }
};
typedef Vec<float, 3> Vec3f;
typedef Vec<unsigned char, 3> Vec3b;
typedef Vec<float, 6> Vec6f;
typedef Vec<float, 4> Vec4f;
typedef Vec<double, 3> Vec3d;

template <class T> struct Point_ {
    T x = 0, y = 0;
    Point_() {}
    Point_(T a, T b) : x(a), y(b) {}
};
typedef Point_<int> Point;
typedef Point_<float> Point2f;
struct Size {
    int width = 0, height = 0;
    Size() {}
    Size(int w, int h) : width(w), height(h) {}
    int area() const { return width * height; }
};
struct Rect {
    int x = 0, y = 0, width = 0, height = 0;
    Rect() {}
    Rect(int a, int b, int w, int h) : x(a), y(b), width(w), height(h) {}
    template <class T> bool contains(const Point_<T>& p) const {
        return x <= p.x && p.x < x + width && y <= p.y && p.y < y + height;
    }
};
struct Scalar {
    double val[4] = {0, 0, 0, 0};
    Scalar() {}
    Scalar(double a, double b = 0, double c = 0, double d = 0) { val[0] = a; val[1] = b; val[2] = c; val[3] = d; }
};

enum { IMREAD_GRAYSCALE = 0, IMREAD_COLOR = 1, IMWRITE_PNG_COMPRESSION = 16, INTER_NEAREST = 0, INTER_LINEAR = 1,
       COLOR_BGR2GRAY = 6, COLOR_GRAY2BGR = 8 };

class Mat {
public:
    int rows = 0, cols = 0;
    uchar* data = nullptr;
    struct Step {
        size_t s[2] = {0, 0};
        size_t operator[](int i) const { return s[i]; }
        operator size_t() const { return s[0]; }
    } step;

    Mat() {}
    Mat(int r, int c, int type) { create(r, c, type); }
    Mat(int r, int c, int type, const Scalar& s) {
        create(r, c, type);
        fill(s);
    }
    Mat(Size sz, int type) { create(sz.height, sz.width, type); }
    Mat(int r, int c, int type, void* ext) {
        type_ = type; rows = r; cols = c; data = static_cast<uchar*>(ext);
        step.s[0] = (size_t)c * elemSize(); step.s[1] = elemSize();
    }

    void create(int r, int c, int type) {
        type_ = type;
        rows = r;
        cols = c;
        const size_t bytes = (size_t)r * c * elemSize();
        store_ = std::make_shared<std::vector<uchar>>(bytes, 0);
        data = store_->data();
        step.s[0] = (size_t)c * elemSize();
        step.s[1] = elemSize();
    }
    static Mat zeros(int r, int c, int type) { return Mat(r, c, type); }
    static Mat zeros(Size sz, int type) { return Mat(sz.height, sz.width, type); }
    static Mat ones(int r, int c, int type) { Mat m(r, c, type); m.fill(Scalar(1, 1, 1, 1)); return m; }

    Mat clone() const {
        Mat m;
        if (data) {
            m.create(rows, cols, type_);
            std::memcpy(m.data, data, (size_t)rows * cols * elemSize());
        }
        return m;
    }
    void release() { store_.reset(); data = nullptr; rows = cols = 0; }
    bool empty() const { return data == nullptr || rows == 0 || cols == 0; }
    Size size() const { return Size(cols, rows); }
    int type() const { return type_; }
    int depth() const { return type_ & 7; }
    int channels() const { return type_channels(type_); }
    size_t elemSize() const { return (size_t)depth_bytes(type_) * type_channels(type_); }
    size_t total() const { return (size_t)rows * cols; }
    bool isContinuous() const { return true; }

    template <class T> T& at(int r, int c) { return reinterpret_cast<T*>(data + (size_t)r * step.s[0])[c]; }
    template <class T> const T& at(int r, int c) const {
        return reinterpret_cast<const T*>(data + (size_t)r * step.s[0])[c];
    }
    template <class T> T& at(int i) { return reinterpret_cast<T*>(data)[i]; }
    template <class T> T* ptr(int r = 0) { return reinterpret_cast<T*>(data + (size_t)r * step.s[0]); }
    template <class T> const T* ptr(int r = 0) const { return reinterpret_cast<const T*>(data + (size_t)r * step.s[0]); }
    uchar* ptr(int r = 0) { return data + (size_t)r * step.s[0]; }

    void copyTo(Mat& dst) const { dst = clone(); }
    void convertTo(Mat& dst, int rtype, double alpha = 1, double beta = 0) const;
    Mat& setTo(const Scalar& s) { fill(s); return *this; }

protected:
    int type_ = CV_8UC1;
    std::shared_ptr<std::vector<uchar>> store_;

    void fill(const Scalar& s) {
        const int cn = channels(), d = depth();
        for (size_t i = 0; i < total(); ++i)
            for (int k = 0; k < cn; ++k) {
                uchar* p = data + i * elemSize() + (size_t)k * depth_bytes(type_);
                const double v = s.val[k < 4 ? k : 3];
                switch (d) {
                    case CV_8U: *p = (uchar)v; break;
                    case CV_32S: *reinterpret_cast<int*>(p) = (int)v; break;
                    case CV_32F: *reinterpret_cast<float*>(p) = (float)v; break;
                    case CV_64F: *reinterpret_cast<double*>(p) = v; break;
                    default: break;
                }
            }
    }
};

template <class T> struct DataType { enum { type = CV_8UC1 }; };
template <> struct DataType<uchar> { enum { type = CV_8UC1 }; };
template <> struct DataType<int> { enum { type = CV_32SC1 }; };
template <> struct DataType<float> { enum { type = CV_32FC1 }; };
template <> struct DataType<double> { enum { type = CV_64FC1 }; };
template <> struct DataType<Vec3b> { enum { type = CV_8UC3 }; };
template <> struct DataType<Vec3f> { enum { type = CV_32FC3 }; };
template <> struct DataType<Vec6f> { enum { type = CV_MAKETYPE(CV_32F, 6) }; };

template <class T>
class Mat_ : public Mat {
public:
    Mat_() { type_ = DataType<T>::type; }
    Mat_(int r, int c) { create(r, c, DataType<T>::type); }
    Mat_(int r, int c, const T& v) {
        create(r, c, DataType<T>::type);
        for (size_t i = 0; i < total(); ++i) reinterpret_cast<T*>(data)[i] = v;
    }
    Mat_(Size sz) { create(sz.height, sz.width, DataType<T>::type); }
    Mat_(const Mat& m) : Mat(m) {}
    Mat_& operator=(const Mat& m) {
        Mat::operator=(m);
        return *this;
    }
    T& operator()(int r, int c) { return at<T>(r, c); }
    const T& operator()(int r, int c) const { return at<T>(r, c); }
    Mat_ clone() const { return Mat_(Mat::clone()); }
};

// defined in oracle/ref_host_driver.cpp (reads <path>.raw)
Mat imread(const std::string& path, int flags = IMREAD_COLOR);

// declared only: not reached from ConfidenceEvaluation or RunFusion
bool imwrite(const std::string& path, const Mat& m, const std::vector<int>& params = std::vector<int>());
void resize(const Mat& src, Mat& dst, Size dsize, double fx = 0, double fy = 0, int interpolation = INTER_LINEAR);
void cvtColor(const Mat& src, Mat& dst, int code);
void Canny(const Mat& src, Mat& edges, double t1, double t2, int aperture = 3, bool l2 = false);
void line(Mat& img, Point a, Point b, const Scalar& color, int thickness = 1, int type = 8, int shift = 0);
void merge(const std::vector<Mat>& mv, Mat& dst);
void merge(const Mat* mv, size_t count, Mat& dst);

class SVD {
public:
    enum { MODIFY_A = 1, NO_UV = 2, FULL_UV = 4 };
    static void compute(const Mat& src, Mat& w, Mat& u, Mat& vt, int flags = 0);
    static void solveZ(const Mat& src, Mat& dst);
};

class Subdiv2D {
public:
    Subdiv2D();
    Subdiv2D(Rect rect);
    void initDelaunay(Rect rect);
    int insert(Point2f pt);
    void insert(const std::vector<Point2f>& pts);
    void getTriangleList(std::vector<Vec6f>& triangleList) const;
};

}  // namespace cv
