// Stand-in declarations for the SZ3-ncp library API that the reference STZ
// sources include (SZ3-ncp itself is not available to this project).
//
// Only the names and signatures the reference translation units mention are
// declared, so that the reference's SZ3-independent templates (split/merge,
// predictors, quantize_range_nodec, planner) compile unmodified. Every body
// here aborts: the oracle never calls into SZ3, it drives the reference's own
// predictor/quantizer functions directly and supplies its own base codec.
//
// This is test infrastructure only (oracle/_ref recipe); nothing in the
// product library includes it.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <utility>
#include <vector>

namespace stz_stub_detail {
[[noreturn]] inline void unavailable(const char* what)
{
    std::fprintf(stderr, "SZ3-ncp stub: %s is not available in the oracle build\n", what);
    std::abort();
}
}  // namespace stz_stub_detail

extern "C" size_t ZSTD_compressBound(size_t srcSize);

namespace SZ3 {

using uchar = unsigned char;

enum ALGO { ALGO_LORENZO_REG, ALGO_INTERP_LORENZO, ALGO_INTERP, ALGO_NOPRED, ALGO_LOSSLESS };
enum EB { EB_ABS, EB_REL, EB_PSNR, EB_L2NORM, EB_ABS_AND_REL, EB_ABS_OR_REL };

struct Config {
    // SZ3's default quantization bin count (radius 32768).
    int quantbinCnt = 65536;
    int cmprAlgo = ALGO_INTERP_LORENZO;
    int errorBoundMode = EB_ABS;
    double absErrorBound = 0.0;
    size_t num = 0;
    Config() = default;
    Config(size_t d0, size_t d1, size_t d2) : num(d0 * d1 * d2) {}
    size_t size_est() const { stz_stub_detail::unavailable("Config::size_est"); }
    void save(uchar*&) const { stz_stub_detail::unavailable("Config::save"); }
    void load(const uchar*&) { stz_stub_detail::unavailable("Config::load"); }
};

template <class T>
inline void write(const T&, uchar*&) { stz_stub_detail::unavailable("SZ3::write"); }
template <class T>
inline void read(T&, const uchar*&, size_t&) { stz_stub_detail::unavailable("SZ3::read"); }

template <class T>
class HuffmanEncoder {
public:
    static void set_forced_marker(size_t, size_t, size_t, size_t) {}
    static void clear_forced_marker() {}
    void preprocess_encode_fast(const T*, size_t, int) { stz_stub_detail::unavailable("HuffmanEncoder::preprocess_encode_fast"); }
    size_t size_est() { stz_stub_detail::unavailable("HuffmanEncoder::size_est"); }
    void save(uchar*&) { stz_stub_detail::unavailable("HuffmanEncoder::save"); }
    void encode_marked_fast(const T*, size_t, uchar*&) { stz_stub_detail::unavailable("HuffmanEncoder::encode_marked_fast"); }
    void postprocess_encode() {}
    void load(const uchar*&, size_t&) { stz_stub_detail::unavailable("HuffmanEncoder::load"); }
    std::vector<T> decode_fast(const uchar*&, size_t) { stz_stub_detail::unavailable("HuffmanEncoder::decode_fast"); }
    template <class Out, class Fn>
    bool decode_marked_transform(const uchar*&, size_t, Out*, Fn&&) { stz_stub_detail::unavailable("HuffmanEncoder::decode_marked_transform"); }
    std::vector<T> decode_marked_chunks_fast(const uchar*&, size_t, const std::vector<size_t>&)
    {
        stz_stub_detail::unavailable("HuffmanEncoder::decode_marked_chunks_fast");
    }
    void postprocess_decode() {}
};

template <class T>
class LinearQuantizer {
public:
    LinearQuantizer() = default;
    LinearQuantizer(double, int) {}
    int quantize_and_overwrite(T&, T) { stz_stub_detail::unavailable("LinearQuantizer::quantize_and_overwrite"); }
    T recover(T, int) { stz_stub_detail::unavailable("LinearQuantizer::recover"); }
    void postcompress_data() {}
    size_t size_est() { stz_stub_detail::unavailable("LinearQuantizer::size_est"); }
    void save(uchar*&) const { stz_stub_detail::unavailable("LinearQuantizer::save"); }
    void load(const uchar*&, size_t&) { stz_stub_detail::unavailable("LinearQuantizer::load"); }
    double get_eb() const { stz_stub_detail::unavailable("LinearQuantizer::get_eb"); }
    std::pair<int, int> get_out_range() const { stz_stub_detail::unavailable("LinearQuantizer::get_out_range"); }
};

class Lossless_zstd {
public:
    size_t compress(const uchar*, size_t, uchar*, size_t) { stz_stub_detail::unavailable("Lossless_zstd::compress"); }
    void decompress(const uchar*, size_t, uchar*&, size_t&) { stz_stub_detail::unavailable("Lossless_zstd::decompress"); }
};

}  // namespace SZ3

template <class T>
char* SZ_compress(SZ3::Config&, T*, size_t&) { stz_stub_detail::unavailable("SZ_compress"); }
template <class T>
void SZ_decompress(SZ3::Config&, char*, size_t, T*) { stz_stub_detail::unavailable("SZ_decompress"); }
