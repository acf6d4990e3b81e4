// Test infrastructure only: decodes a Dirac bitstream with the reference decoder through its
// own public C API (libdirac_decoder/dirac_parser.h: dirac_decoder_init, dirac_buffer,
// dirac_parse, dirac_set_buf, dirac_decoder_close), returning the decoded frames by frame
// number, so that the tests can pin decoding against the reference decoder itself.  Linked
// into oracle/_ref/libdirac_ref.so.

#include <cstring>
#include <vector>

#include <libdirac_decoder/dirac_parser.h>

extern "C" {

// Decodes `bytes` bytes of a stream of 8-bit pictures w x h (chroma cw x ch).  frames receives
// up to nframes frames (Y then U then V, dense, frame after frame) at their frame numbers;
// got[k] = 1 for each frame k delivered.  Returns the number of frames delivered, or -1 when
// the decoder reports an invalid stream or a different picture size.
int ref_decode_stream(const unsigned char* stream, long long bytes, int w, int h, int cw, int ch, int nframes,
                      unsigned char* frames, int* got) {
    dirac_decoder_t* dec = dirac_decoder_init(0);
    if (!dec) return -1;
    const size_t fsize = (size_t)w * h + 2 * (size_t)cw * ch;
    std::vector<unsigned char> y((size_t)w * h), u((size_t)cw * ch), v((size_t)cw * ch);
    for (int k = 0; k < nframes; ++k) got[k] = 0;
    int delivered = 0, rc = 0;
    bool fed = false, done = false;
    // every parse call consumes data or changes state, so a bounded number of calls suffices
    for (long long guard = 0; guard < 64LL * nframes + 1024 && !done; ++guard) {
        switch (dirac_parse(dec)) {
            case STATE_BUFFER:
                if (fed) {
                    done = true;  // the whole stream has been consumed
                    break;
                }
                dirac_buffer(dec, const_cast<unsigned char*>(stream), const_cast<unsigned char*>(stream) + bytes);
                fed = true;
                break;
            case STATE_SEQUENCE: {
                if ((int)dec->src_params.width != w || (int)dec->src_params.height != h ||
                    (int)dec->src_params.chroma_width != cw || (int)dec->src_params.chroma_height != ch) {
                    rc = -1;
                    done = true;
                    break;
                }
                unsigned char* buf[3] = {y.data(), u.data(), v.data()};
                dirac_set_buf(dec, buf, nullptr);
                break;
            }
            case STATE_PICTURE_AVAIL: {
                const int k = (int)dec->frame_num;
                if (k >= 0 && k < nframes) {
                    unsigned char* dst = frames + (size_t)k * fsize;
                    std::memcpy(dst, y.data(), y.size());
                    std::memcpy(dst + y.size(), u.data(), u.size());
                    std::memcpy(dst + y.size() + u.size(), v.data(), v.size());
                    if (!got[k]) ++delivered;
                    got[k] = 1;
                }
                break;
            }
            case STATE_SEQUENCE_END:
                done = true;
                break;
            case STATE_INVALID:
                rc = -1;
                done = true;
                break;
            default:
                break;
        }
    }
    dirac_decoder_close(dec);
    return rc ? rc : delivered;
}

}  // extern "C"
