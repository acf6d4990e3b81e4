// Test infrastructure only: an extern "C" stage driver over the reference codec's own
// classes, compiled together with the reference sources into oracle/_ref/libdirac_ref.so.
// The tests and the golden-fixture generator call it to run the reference itself on the
// same bytes the CUDA path sees.  Nothing in the product links or loads this file.
//
// Every array crossing this boundary is dense row-major with the stated width as stride.

#include <cstring>
#include <vector>

#include <libdirac_common/common.h>
#include <libdirac_common/wavelet_utils.h>
#include <libdirac_common/upconvert.h>
#include <libdirac_motionest/downconvert.h>

using namespace dirac;

namespace {

void fill_pic(PicArray& a, const short* src) {
    for (int j = 0; j < a.LengthY(); ++j)
        std::memcpy(&a[j][0], src + (size_t)j * a.LengthX(), sizeof(short) * a.LengthX());
}

void read_pic(const PicArray& a, short* dst) {
    for (int j = 0; j < a.LengthY(); ++j)
        std::memcpy(dst + (size_t)j * a.LengthX(), &a[j][0], sizeof(short) * a.LengthX());
}

template <class A, class T>
void fill_arr(A& a, const T* src) {
    for (int j = 0; j < a.LengthY(); ++j)
        std::memcpy(&a[j][0], src + (size_t)j * a.LengthX(), sizeof(T) * a.LengthX());
}

template <class A, class T>
void read_arr(const A& a, T* dst) {
    for (int j = 0; j < a.LengthY(); ++j)
        std::memcpy(dst + (size_t)j * a.LengthX(), &a[j][0], sizeof(T) * a.LengthX());
}

}  // namespace

extern "C" {

// WaveletTransform(depth, filter).Transform(FORWARD, pic, coeff)
// (libdirac_common/wavelet_utils.cpp:440-466).  pic is h x w int16, coeff is ch x cw int32
// (the padded size, a multiple of 2^depth).  Returns 0, or -1 on an exception.
int ref_dwt_forward(int filter, int depth, const short* pic, int w, int h, int* coeff, int cw, int ch) {
    try {
        PicArray p(h, w);
        fill_pic(p, pic);
        CoeffArray c(ch, cw);
        WaveletTransform wt(depth, (WltFilter)filter);
        wt.Transform(FORWARD, p, c);
        read_arr(c, coeff);
        return 0;
    } catch (...) {
        return -1;
    }
}

// WaveletTransform(depth, filter).Transform(BACKWARD, pic, coeff)
// (wavelet_utils.cpp:467-484): synthesises coeff in place and writes the truncated
// int16 picture.  coeff is read and overwritten.
int ref_dwt_backward(int filter, int depth, int* coeff, int cw, int ch, short* pic, int w, int h) {
    try {
        PicArray p(h, w);
        CoeffArray c(ch, cw);
        fill_arr(c, coeff);
        WaveletTransform wt(depth, (WltFilter)filter);
        wt.Transform(BACKWARD, p, c);
        read_arr(c, coeff);
        read_pic(p, pic);
        return 0;
    } catch (...) {
        return -1;
    }
}

// UpConverter(min,max,orig_w,orig_h).DoUpConverter (libdirac_common/upconvert.cpp:55-145).
// up is (2h) x (2w).
int ref_upconvert(const short* pic, int w, int h, int depth, short* up) {
    try {
        PicArray p(h, w);
        fill_pic(p, pic);
        PicArray u(2 * h, 2 * w);
        u.Fill(0);
        UpConverter uc(-(1 << (depth - 1)), (1 << (depth - 1)) - 1, w, h);
        uc.DoUpConverter(p, u);
        read_pic(u, up);
        return 0;
    } catch (...) {
        return -1;
    }
}

// DownConverter::DoDownConvert (libdirac_motionest/downconvert.cpp:51-147); out is
// (h/2) x (w/2), as PixelMatcher::MakePicHierarchy sizes it (pixel_match.cpp:158-167).
int ref_downconvert(const short* pic, int w, int h, short* out) {
    try {
        PicArray p(h, w);
        fill_pic(p, pic);
        PicArray o(h / 2, w / 2);
        DownConverter dc;
        dc.DoDownConvert(p, o);
        read_pic(o, out);
        return 0;
    } catch (...) {
        return -1;
    }
}

}  // extern "C"
