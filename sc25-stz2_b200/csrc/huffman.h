// Host-side launchers of the chunked canonical-Huffman kernels (huffman.cu).
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

#include "stz_internal.h"

namespace stz {

// A chunk holding unpredictable values and where its values sit in the
// stream's compact list.
struct UnpredWork {
    uint32_t stream;
    uint32_t chunk;
    uint64_t list_off;
    uint64_t count;  // values of this chunk in the list
};

// Dense code table per stream (2*radius entries): code << 5 | length.
void launch_expand_codebook(const StreamDesc* sd, int nstreams, const uint16_t* cb_sym, const uint8_t* cb_len,
                            uint32_t* ctab, cudaStream_t st);
// Run-symbol counts per stream (streams with run_n > 0): stats[s * kRunStats]
// gets the centre codes left as single symbols, stats[s * kRunStats + 1 + i]
// the uses of run slot i. stats must be zeroed.
constexpr int kRunStats = 64;
// Per stream: the bits of a run of r centre codes, r < kRunBitsStride
// (launch_run_bits; planes of up to 1024 codes).
constexpr uint32_t kRunBitsStride = 1025;
void launch_run_stats(const CtaWork* work, const uint32_t* chunk_ids, int nwork, const StreamDesc* sd,
                      const uint16_t* codes, unsigned long long* stats, cudaStream_t st);
// Bits of a run of r centre codes per stream (rbits: nstreams x
// kRunBitsStride bytes), from the stream's code table (after
// launch_expand_codebook); streams with runs and planes of up to 1024 codes.
void launch_run_bits(const StreamDesc* sd, int nstreams, const uint32_t* ctab, uint8_t* rbits, cudaStream_t st);
void launch_sub_bits(const CtaWork* work, const uint32_t* chunk_ids, int nwork, const StreamDesc* sd,
                     const uint16_t* codes, const uint32_t* ctab, const uint8_t* rbits, uint32_t* sub_bits,
                     cudaStream_t st);
// Plane bit offsets, chunk word offsets and stream word counts from the
// plane bit counts; clears every plane's boundary words (max_chunks: the
// most chunks of any stream).
void launch_scan_streams(const StreamDesc* sd, int nstreams, uint32_t max_chunks, const uint32_t* sub_bits,
                         uint32_t* sub_off, uint64_t* chunk_word_off, uint64_t* stream_words, uint32_t* payload,
                         cudaStream_t st);
void launch_encode(const CtaWork* work, const uint32_t* chunk_ids, int nwork, const StreamDesc* sd,
                   const uint16_t* codes, const uint32_t* ctab, const uint8_t* rbits, const uint32_t* sub_bits,
                   const uint32_t* sub_off, const uint64_t* chunk_word_off, uint32_t* payload, cudaStream_t st);
void launch_decode(const CtaWork* work, const uint32_t* chunk_ids, int nwork, const StreamDesc* sd,
                   const uint16_t* cb_sym, const void* tables, const uint32_t* sub_off, const uint64_t* chunk_word_off,
                   const uint32_t* payload, uint16_t* codes, cudaStream_t st);
// Decode tables of every stream (read by the decoders): decode_tables_bytes()
// each, stream i at byte i * decode_tables_bytes() of `tables`.
size_t decode_tables_bytes();
// Mean payload bits per plane above which launch_decode decodes a stream one
// thread per plane instead of a lane group per plane, in launches of at least 128
// work items and for streams of at least 16384 planes (STZ_DECODE_SEQ_BITS
// overrides the built-in 2048).
uint32_t decode_seq_bits();
void launch_build_tables(const StreamDesc* sd, int nstreams, const uint16_t* cb_sym, const uint8_t* cb_len,
                         void* tables, cudaStream_t st);
// The payload words of streams [s0, s1) back to back in stream order into dst
// (each stream's count from stream_words, as k_scan_stream leaves it), so a
// group of small streams goes to the host in one transfer.
void launch_pack_streams(const StreamDesc* sd, const uint64_t* stream_words, int s0, int s1, const uint32_t* payload,
                         uint32_t* dst, cudaStream_t st);
template <typename T>
void launch_unpred_move(bool gather, const UnpredWork* work, int nwork, const StreamDesc* sd, const uint16_t* codes,
                        T* dense, T* list, cudaStream_t st);

// Persistent variants for captured graphs: `grid` CTAs walk the lists of a
// batch held in device memory (BatchHdr at meta: n_work/o_work/o_ids,
// n_uwork/o_uwork).
void launch_decode_dyn(int grid, const uint8_t* meta, const StreamDesc* sd, const uint16_t* cb_sym,
                       const void* tables, const uint32_t* sub_off, const uint64_t* chunk_word_off,
                       const uint32_t* payload, uint16_t* codes, cudaStream_t st);
template <typename T>
void launch_unpred_scatter_dyn(int grid, const uint8_t* meta, const StreamDesc* sd, const uint16_t* codes, T* dense,
                               T* list, cudaStream_t st);

}  // namespace stz
