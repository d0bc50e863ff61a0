// Bitshuffle/LZ4 frames decoded on the device in front of the gather
// (Cuda1dPlan::integrate_bslz4 and Cuda2dPlan::integrate_bslz4,
// src/integration/cuda.rs:554-564 and :758-767), and a host encoder that
// writes the same chunks.
//
// Chunk layout (HDF5's bitshuffle filter with LZ4): a big-endian u64 of the
// frame's bytes and a big-endian u32 block size in bytes (0 means 8192); then,
// for every full block of block/elem elements and for the remainder rounded
// down to a multiple of 8 elements, a big-endian u32 compressed length and an
// LZ4 block holding the block's elements bitshuffled; the last (< 8) elements
// follow verbatim. Bitshuffled means: bit plane p (bit p of an element, least
// significant first) holds n/8 bytes, bit i of byte k being bit p of element
// 8k + i.
//
// Host side. Every chunk's 12-byte header is checked before any device work;
// frames are then cut into batches, and while the device decodes and
// integrates one batch the host walks the next batch's block lengths (the
// walk is a chain of dependent reads, so frames are walked by several
// threads) into one 16-byte descriptor per block, with the bounds the
// reference checks (src/integration/cuda/device.rs:2056-2178). Compressed
// bytes go to the device on a copy stream into two alternating slots.
//
// Device decoding: one warp per block. The warp first stages the block's
// compressed bytes at the end of its shared-memory region with 16-byte loads
// (many in flight), so the sequential parse reads shared memory, and decodes
// in place towards the region's start. Every lane
// parses the same token and length bytes (broadcast reads, no shuffles), the
// warp copies a sequence's literals, and copies its match in one parallel
// pass — byte i of a match at distance d is the already decoded byte at
// start - d + (i mod d), so no lane reads a byte written in the same pass,
// whatever d. Each lane then takes one 32-bit word of every bit plane (32
// consecutive elements), transposes the 32 x 32 bit matrix in registers and
// stores its 32 elements into the frame buffer the gather reads.
#include <algorithm>
#include <cstring>
#include <thread>
#include <type_traits>

#include "dg_internal.h"

namespace dg {
namespace {

constexpr int kMaxBlockBytes = 48 * 1024;  // largest block the decoder stages
constexpr size_t kSmemPerSm = 227 * 1024;  // dynamic shared memory one CTA may use

// Descriptor: {first compressed byte in the batch, compressed bytes (bit 31:
// verbatim tail), first element in the batch's frame buffer, decoded bytes}.
using BlockDesc = uint4;

// Shared memory one warp decodes a block of at most `block` bytes in. The
// compressed bytes are staged at the end of the region and decoded in place
// towards its start (see k_bslz4_decode); the region holds the decoded block,
// the LZ4 worst-case expansion (block / 255 + 16) and slack for the staging's
// 16-byte alignment and the in-place read-ahead.
uint32_t region_bytes(uint32_t block) { return (block + block / 255 + 96 + 15) / 16 * 16; }

}  // namespace

// In-place transpose of a 32 x 32 bit matrix held as 32 words (row r = a[r],
// column c = bit c): afterwards bit r of a[c] is the former bit c of a[r].
// Recursive block swap: at step j the off-diagonal j x j blocks of every
// 2j x 2j tile trade places.
__host__ __device__ __forceinline__ void transpose32(uint32_t (&a)[32]) {
    const uint32_t masks[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
    for (int s = 0; s < 5; ++s) {
        const int j = 16 >> s;
        const uint32_t m = masks[s];
#pragma unroll
        for (int r = 0; r < 32; ++r) {
            if (r & j) continue;
            const uint32_t t = ((a[r] >> j) ^ a[r + j]) & m;
            a[r] ^= t << j;
            a[r + j] ^= t;
        }
    }
}

namespace {

// One warp per descriptor; blockDim.x / 32 warps per CTA, each with `region`
// bytes of dynamic shared memory.
//
// In-place decoding: the compressed block (clen bytes) is staged at the end
// of the warp's region, starting at p >= region - 31 - clen, and decoded from
// position 0 upwards. For any prefix of a valid LZ4 block, decoded bytes
// minus consumed bytes is at most total - clen + total / 255 + 2 (a suffix of
// the block consumes at most its literals, a token per 255 of them and one
// last token more than it produces; every match produces more than its 3+
// bytes of token and offset). With region >= total + total / 255 + 96 the
// write position therefore never passes the read position p + ipos, and a
// match never overwrites bytes not yet read. A corrupt block may break that
// order; it then decodes to garbage or is rejected, with every access still
// inside the warp's region.
template <int E>
__global__ void __launch_bounds__(128)
    k_bslz4_decode(const uint8_t *__restrict__ comp, const BlockDesc *__restrict__ desc,
                   uint32_t n_blocks, uint32_t region, void *__restrict__ out,
                   int *__restrict__ err) {
    using T = typename std::conditional<E == 2, uint16_t, uint32_t>::type;
    extern __shared__ __align__(16) uint8_t sm_blocks[];
    // lane % d and 32 % d for match distances d = 1..32
    __shared__ uint8_t mod_lane[32 * 32], mod_32[32];
    for (int i = threadIdx.x; i < 32 * 32; i += blockDim.x) mod_lane[i] = uint8_t((i & 31) % ((i >> 5) + 1));
    if (threadIdx.x < 32) mod_32[threadIdx.x] = uint8_t(32 % (threadIdx.x + 1));
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t b = blockIdx.x * (blockDim.x >> 5) + warp;
    if (b >= n_blocks) return;
    const BlockDesc d = desc[b];
    T *dst = static_cast<T *>(out) + d.z;
    if (d.y & 0x80000000u) {  // verbatim tail
        const uint8_t *ip = comp + d.x;
        uint8_t *db = reinterpret_cast<uint8_t *>(dst);
        for (uint32_t i = lane; i < d.w; i += 32) db[i] = __ldg(ip + i);
        return;
    }
    const uint32_t clen = d.y, total = d.w;
    uint8_t *buf = sm_blocks + size_t(warp) * region;
    // Stage the compressed bytes at the region's end: 16-byte loads from the
    // aligned start below them to the aligned end above them (both inside the
    // batch's slot, which starts and ends on 256-byte boundaries), eight per
    // lane in flight; p has the source's alignment modulo 16.
    const uintptr_t g = reinterpret_cast<uintptr_t>(comp + d.x);
    const uint32_t p0 = region - 16 - clen;
    const uint32_t p = p0 - ((p0 - uint32_t(g & 15)) & 15u);
    {
        const uint4 *gv = reinterpret_cast<const uint4 *>(g & ~uintptr_t(15));
        const uint32_t nvec = uint32_t((g & 15) + clen + 15) / 16;
        uint4 *sv = reinterpret_cast<uint4 *>(buf + (p - uint32_t(g & 15)));
        for (uint32_t v0 = 0; v0 < nvec; v0 += 256) {
            uint4 r[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const uint32_t v = v0 + u * 32 + lane;
                if (v < nvec) r[u] = __ldg(gv + v);
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const uint32_t v = v0 + u * 32 + lane;
                if (v < nvec) sv[v] = r[u];
            }
        }
        __syncwarp();
    }
    const uint8_t *ip = buf + p;
    uint32_t ipos = 0, opos = 0;
    bool ok = true;
    // Every bound below is uniform across the warp (all lanes parse the same
    // bytes), and every loop advances ipos or opos within clen and total.
    while (ipos < clen) {
        const uint32_t token = ip[ipos++];
        uint32_t lit = token >> 4;
        if (lit == 15) {
            uint32_t s;
            do {
                if (ipos >= clen) {
                    ok = false;
                    break;
                }
                s = ip[ipos++];
                lit += s;
            } while (s == 255 && lit <= total);
        }
        if (!ok || lit > clen - ipos || lit > total - opos) {
            ok = false;
            break;
        }
        // Literals, 32 at a time; the source may lie just above the
        // destination, so every lane loads before any lane stores.
        for (uint32_t i0 = 0; i0 < lit; i0 += 32) {
            const uint32_t i = i0 + lane;
            const uint8_t v = i < lit ? ip[ipos + i] : 0;
            __syncwarp();
            if (i < lit) buf[opos + i] = v;
        }
        ipos += lit;
        opos += lit;
        if (ipos == clen) break;  // the last sequence has literals only
        if (clen - ipos < 2) {
            ok = false;
            break;
        }
        const uint32_t offset = uint32_t(ip[ipos]) | (uint32_t(ip[ipos + 1]) << 8);
        ipos += 2;
        uint32_t mlen = (token & 15u) + 4u;
        if ((token & 15u) == 15u) {
            uint32_t s;
            do {
                if (ipos >= clen) {
                    ok = false;
                    break;
                }
                s = ip[ipos++];
                mlen += s;
            } while (s == 255 && mlen <= total);
        }
        if (!ok || offset == 0 || offset > opos || mlen > total - opos) {
            ok = false;
            break;
        }
        __syncwarp();  // literals of every lane visible before the match reads them
        // Byte i of the match is the decoded byte at from + (i mod offset),
        // before the match: r walks i mod offset in steps of 32.
        const uint8_t *from = buf + (opos - offset);
        uint8_t *to = buf + opos;
        uint32_t r, step;
        if (offset > 32) {
            r = uint32_t(lane);
            step = 32;
        } else {
            r = mod_lane[(offset - 1) * 32 + lane];
            step = mod_32[offset - 1];
        }
        for (uint32_t i = lane; i < mlen; i += 32) {
            to[i] = from[r];
            r += step;
            if (r >= offset) r -= offset;
        }
        opos += mlen;
        __syncwarp();
    }
    if (!ok || opos != total) {
        if (lane == 0) atomicExch(err, 1);
        return;
    }
    __syncwarp();
    const uint32_t n = total / E, plane = n / 8;
    if (n % 32 == 0) {
        const uint32_t words = n / 32;
        for (uint32_t w0 = 0; w0 < words; w0 += 32) {
            const uint32_t w = w0 + lane;
            if (w >= words) break;
            uint32_t a[32];
#pragma unroll
            for (int p = 0; p < 32; ++p)
                a[p] = p < 8 * E ? *reinterpret_cast<const uint32_t *>(buf + p * plane + 4 * w) : 0u;
            transpose32(a);
            T *o = dst + 32 * w;
            if (E == 4) {
                if ((d.z & 3) == 0) {
#pragma unroll
                    for (int k = 0; k < 8; ++k)
                        reinterpret_cast<uint4 *>(o)[k] =
                            make_uint4(a[4 * k], a[4 * k + 1], a[4 * k + 2], a[4 * k + 3]);
                } else {
#pragma unroll
                    for (int k = 0; k < 32; ++k) o[k] = T(a[k]);
                }
            } else {
                if ((d.z & 7) == 0) {
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        reinterpret_cast<uint4 *>(o)[k] = make_uint4(
                            a[8 * k] | (a[8 * k + 1] << 16), a[8 * k + 2] | (a[8 * k + 3] << 16),
                            a[8 * k + 4] | (a[8 * k + 5] << 16), a[8 * k + 6] | (a[8 * k + 7] << 16));
                } else {
#pragma unroll
                    for (int k = 0; k < 32; ++k) o[k] = T(a[k]);
                }
            }
        }
    } else {
        // A block of n = 8, 16 or 24 mod 32 elements (remainder blocks, odd
        // block sizes): element e gathers its bits from the planes' bytes.
        for (uint32_t e = lane; e < n; e += 32) {
            uint32_t v = 0;
#pragma unroll
            for (int p = 0; p < 8 * E; ++p)
                v |= uint32_t((buf[p * plane + e / 8] >> (e % 8)) & 1u) << p;
            dst[e] = T(v);
        }
    }
}

uint64_t rd_be64(const uint8_t *p) {
    uint64_t v = 0;
    for (int i = 0; i < 8; ++i) v = (v << 8) | p[i];
    return v;
}
uint32_t rd_be32(const uint8_t *p) {
    return (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) | (uint32_t(p[2]) << 8) | p[3];
}

// A chunk's header: its block size and the number of descriptors it yields.
struct ChunkHead {
    uint32_t block = 0;
    uint32_t n_desc = 0;
};

ChunkHead check_header(const uint8_t *c, int64_t len, int64_t f, int64_t npix, int elem) {
    const std::string where = "frame " + std::to_string(f) + ": ";
    const uint64_t frame_bytes = uint64_t(npix) * elem;
    if (len < 12)
        fail(DG_INVALID_INPUT, where + "Bitshuffle/LZ4 chunk shorter than its 12-byte header");
    if (rd_be64(c) != frame_bytes)
        fail(DG_INVALID_INPUT, where + "Bitshuffle/LZ4 chunk uncompressed size " +
                                   std::to_string(rd_be64(c)) + " does not match plan frame size " +
                                   std::to_string(frame_bytes) + " bytes");
    int64_t block = rd_be32(c + 8);
    if (block == 0) block = 8192;
    if (block > kMaxBlockBytes || block % (8 * elem))
        fail(DG_INVALID_INPUT, where + "unsupported Bitshuffle/LZ4 block size " +
                                   std::to_string(block) + " bytes");
    const int64_t be = block / elem, rem = npix % be;
    ChunkHead h;
    h.block = uint32_t(block);
    h.n_desc = uint32_t(npix / be + (rem / 8 > 0 ? 1 : 0) + (rem % 8 > 0 ? 1 : 0));
    return h;
}

// Writes the h.n_desc descriptors of one chunk (frame `f` of the call, `slot`
// of its batch, its bytes at `base` of the batch's compressed buffer).
void walk_blocks(const uint8_t *c, int64_t len, int64_t f, int64_t slot, uint64_t base,
                 int64_t npix, int elem, const ChunkHead &h, BlockDesc *out) {
    const int64_t be = h.block / elem, n_full = npix / be, rem = npix % be;
    const int64_t rem_comp = rem / 8 * 8, tail = rem % 8;
    const uint64_t first = uint64_t(slot) * uint64_t(npix);
    auto bad = [&](const std::string &what) {
        fail(DG_INVALID_INPUT, "frame " + std::to_string(f) + ": " + what);
    };
    int64_t off = 12;
    for (int64_t k = 0; k <= n_full; ++k) {
        const int64_t elems = k < n_full ? be : rem_comp;
        if (elems == 0) break;
        if (off + 4 > len) bad("truncated Bitshuffle/LZ4 block header");
        const int64_t clen = rd_be32(c + off);
        off += 4;
        const int64_t ub = elems * elem;
        if (clen > ub + ub / 255 + 16)
            bad("Bitshuffle/LZ4 compressed block length " + std::to_string(clen) +
                " exceeds the LZ4 bound " + std::to_string(ub + ub / 255 + 16));
        if (off + clen > len) bad("truncated Bitshuffle/LZ4 block payload");
        *out++ = make_uint4(uint32_t(base + uint64_t(off)), uint32_t(clen),
                            uint32_t(first + uint64_t(k * be)), uint32_t(ub));
        off += clen;
    }
    if (tail) {
        const int64_t raw = tail * elem;
        if (off + raw > len) bad("truncated Bitshuffle/LZ4 tail bytes");
        *out++ = make_uint4(uint32_t(base + uint64_t(off)), 0x80000000u | uint32_t(raw),
                            uint32_t(first + uint64_t(n_full * be + rem_comp)), uint32_t(raw));
    }
}

// ---------------------------------------------------------------- encoder

void bitshuffle(const uint8_t *in, int64_t count, int elem, uint8_t *out) {
    const int64_t plane = count / 8;
    for (int64_t g = 0; g < plane; ++g) {
        // 8 elements -> one byte of each of the 8*elem planes
        for (int byte = 0; byte < elem; ++byte) {
            uint64_t x = 0;
            for (int i = 0; i < 8; ++i) x |= uint64_t(in[(8 * g + i) * elem + byte]) << (8 * i);
            // 8 x 8 bit transpose: bit b of byte i -> bit i of byte b
            uint64_t t = (x ^ (x >> 7)) & 0x00AA00AA00AA00AAull;
            x ^= t ^ (t << 7);
            t = (x ^ (x >> 14)) & 0x0000CCCC0000CCCCull;
            x ^= t ^ (t << 14);
            t = (x ^ (x >> 28)) & 0x00000000F0F0F0F0ull;
            x ^= t ^ (t << 28);
            for (int bit = 0; bit < 8; ++bit)
                out[(8 * byte + bit) * plane + g] = uint8_t(x >> (8 * bit));
        }
    }
}

void put_len(std::vector<uint8_t> &o, int64_t n) {
    while (n >= 255) {
        o.push_back(255);
        n -= 255;
    }
    o.push_back(uint8_t(n));
}

// One LZ4 block: greedy matching through a hash of the next four bytes, with
// the format's end conditions (the last 5 bytes are literals, no match starts
// within the last 12).
void lz4_compress(const uint8_t *src, int64_t n, std::vector<int32_t> &table,
                  std::vector<uint8_t> &o) {
    std::fill(table.begin(), table.end(), -1);
    int64_t anchor = 0, i = 0;
    auto read32 = [&](int64_t p) {
        uint32_t v;
        std::memcpy(&v, src + p, 4);
        return v;
    };
    auto emit = [&](int64_t lit_end, int64_t offset, int64_t mlen) {
        const int64_t lit = lit_end - anchor;
        o.push_back(uint8_t((std::min<int64_t>(lit, 15) << 4) |
                            (mlen ? std::min<int64_t>(mlen - 4, 15) : 0)));
        if (lit >= 15) put_len(o, lit - 15);
        o.insert(o.end(), src + anchor, src + lit_end);
        if (!mlen) return;
        o.push_back(uint8_t(offset & 255));
        o.push_back(uint8_t(offset >> 8));
        if (mlen - 4 >= 15) put_len(o, mlen - 4 - 15);
    };
    const int64_t last_start = n - 12, match_end = n - 5;
    while (i < last_start) {
        const uint32_t seq = read32(i);
        const uint32_t h = (seq * 2654435761u) >> 20;  // 12-bit hash
        const int64_t ref = table[h];
        table[h] = int32_t(i);
        if (ref >= 0 && i - ref <= 65535 && read32(ref) == seq) {
            int64_t m = 4;
            while (i + m < match_end && src[ref + m] == src[i + m]) ++m;
            emit(i, i - ref, m);
            i += m;
            anchor = i;
        } else {
            ++i;
        }
    }
    emit(n, 0, 0);
}

void record(EventPool &p, cudaStream_t s, bool begin) {
    if (begin) {
        if (p.used == p.events.size()) {
            std::pair<cudaEvent_t, cudaEvent_t> e{};
            DG_CUDA(cudaEventCreate(&e.first));
            DG_CUDA(cudaEventCreate(&e.second));
            p.events.push_back(e);
        }
        DG_CUDA(cudaEventRecord(p.events[p.used++].first, s));
    } else {
        DG_CUDA(cudaEventRecord(p.events[p.used - 1].second, s));
    }
}

template <typename F>
dg_status guarded(F &&f) {
    try {
        f();
        return DG_OK;
    } catch (const Error &e) {
        set_last_error(e.message);
        return e.status;
    } catch (const std::bad_alloc &) {
        set_last_error("host allocation failed");
        return DG_DEVICE;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return DG_DEVICE;
    }
}

// Runs body(k) for k in [0, n) on up to `threads` threads (the caller's
// included); the first error by index is rethrown on the caller's thread.
template <typename F>
void parallel_for(int64_t n, int threads, F &&body) {
    threads = int(std::max<int64_t>(1, std::min<int64_t>(threads, n)));
    if (threads == 1) {
        for (int64_t k = 0; k < n; ++k) body(k);
        return;
    }
    struct Failure {
        bool set = false;
        dg_status status = DG_OK;
        std::string message;
    };
    std::vector<Failure> errs(static_cast<size_t>(n));
    auto run = [&](int t) {
        for (int64_t k = t; k < n; k += threads) {
            Failure &slot = errs[size_t(k)];
            try {
                body(k);
            } catch (const Error &e) {
                slot.set = true;
                slot.status = e.status;
                slot.message = e.message;
            } catch (const std::exception &e) {
                slot.set = true;
                slot.status = DG_DEVICE;
                slot.message = e.what();
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(run, t);
    run(0);
    for (auto &th : pool) th.join();
    for (const Failure &e : errs)
        if (e.set) fail(e.status, e.message);
}

}  // namespace

void bslz4_release(dg_plan *plan) {
    plan->stage_comp.release();
    plan->stage_desc.release();
    plan->decode_events.destroy();
    for (int k = 0; k < 2; ++k) {
        if (plan->bs_copied[k]) cudaEventDestroy(plan->bs_copied[k]);
        if (plan->bs_decoded[k]) cudaEventDestroy(plan->bs_decoded[k]);
        plan->bs_copied[k] = plan->bs_decoded[k] = nullptr;
    }
    if (plan->copy_stream) cudaStreamDestroy(plan->copy_stream);
    plan->copy_stream = nullptr;
}

void ensure_copy_pipeline(dg_plan *plan) {
    if (!plan->copy_stream)
        DG_CUDA(cudaStreamCreateWithFlags(&plan->copy_stream, cudaStreamNonBlocking));
    for (int k = 0; k < 2; ++k) {
        if (!plan->bs_copied[k])
            DG_CUDA(cudaEventCreateWithFlags(&plan->bs_copied[k], cudaEventDisableTiming));
        if (!plan->bs_decoded[k])
            DG_CUDA(cudaEventCreateWithFlags(&plan->bs_decoded[k], cudaEventDisableTiming));
    }
}

}  // namespace dg

extern "C" {

int64_t dg_bslz4_bound(int64_t n_elems, int32_t elem_bytes, int32_t block_bytes) {
    if (n_elems < 0 || (elem_bytes != 2 && elem_bytes != 4) || block_bytes < 0) return -1;
    const int64_t block = block_bytes ? block_bytes : 8192;
    const int64_t bytes = n_elems * elem_bytes;
    return 12 + bytes + (bytes / block + 2) * (4 + block / 255 + 16);
}

dg_status dg_bslz4_compress(const void *frame, int64_t n_elems, int32_t elem_bytes,
                            int32_t block_bytes, void *out, int64_t capacity, int64_t *out_bytes) {
    using namespace dg;
    return guarded([&] {
        if ((!frame && n_elems) || !out || !out_bytes || n_elems < 0)
            fail(DG_INVALID_INPUT, "frame, out and out_bytes must not be NULL");
        if (elem_bytes != 2 && elem_bytes != 4)
            fail(DG_INVALID_INPUT, "Bitshuffle/LZ4 chunks hold 2- or 4-byte elements");
        const int64_t block = block_bytes ? block_bytes : 8192;
        if (block <= 0 || block > kMaxBlockBytes || block % (8 * elem_bytes))
            fail(DG_INVALID_INPUT,
                 "block size must be a positive multiple of 8 elements, at most 48 KiB");
        const uint8_t *raw = static_cast<const uint8_t *>(frame);
        std::vector<uint8_t> o;
        o.reserve(size_t(std::max<int64_t>(0, std::min<int64_t>(capacity, n_elems * elem_bytes + 64))));
        const uint64_t total = uint64_t(n_elems) * elem_bytes;
        for (int i = 7; i >= 0; --i) o.push_back(uint8_t(total >> (8 * i)));
        for (int i = 3; i >= 0; --i) o.push_back(uint8_t(uint32_t(block_bytes) >> (8 * i)));
        const int64_t be = block / elem_bytes, n_full = n_elems / be, rem = n_elems % be;
        const int64_t rem_comp = rem / 8 * 8, tail = rem % 8;
        std::vector<uint8_t> shuf(static_cast<size_t>(block));
        std::vector<int32_t> table(1 << 12);
        for (int64_t k = 0; k <= n_full; ++k) {
            const int64_t elems = k < n_full ? be : rem_comp;
            if (elems == 0) break;
            bitshuffle(raw + k * be * elem_bytes, elems, elem_bytes, shuf.data());
            const size_t at = o.size();
            o.resize(at + 4);
            lz4_compress(shuf.data(), elems * elem_bytes, table, o);
            const uint32_t clen = uint32_t(o.size() - at - 4);
            for (int i = 0; i < 4; ++i) o[at + size_t(i)] = uint8_t(clen >> (8 * (3 - i)));
        }
        if (tail)
            o.insert(o.end(), raw + (n_full * be + rem_comp) * elem_bytes,
                     raw + n_elems * elem_bytes);
        if (int64_t(o.size()) > capacity)
            fail(DG_INVALID_INPUT, "output capacity " + std::to_string(capacity) +
                                       " too small for " + std::to_string(o.size()) + " bytes");
        std::memcpy(out, o.data(), o.size());
        *out_bytes = int64_t(o.size());
    });
}

dg_status dg_integrate_bslz4(dg_plan *plan, const void *const *chunks, const int64_t *chunk_bytes,
                             int64_t n_frames, int32_t dtype, uint32_t flags, double *oi,
                             double *os, double *od) {
    using namespace dg;
    const dg_status st = guarded([&] {
        if (!plan) fail(DG_INVALID_INPUT, "plan must not be NULL");
        if (dtype != DG_U16 && dtype != DG_U32 && dtype != DG_I32)
            fail(DG_INVALID_INPUT, "Bitshuffle/LZ4 frames must be uint16, uint32 or int32");
        if (flags & ~uint32_t(DG_ERRORS | DG_AZIMUTHAL_STD)) fail(DG_INVALID_INPUT, "unknown flags");
        if (n_frames < 0) fail(DG_INVALID_INPUT, "frame count must not be negative");
        if (n_frames == 0) return;
        if (!chunks || !chunk_bytes) fail(DG_INVALID_INPUT, "chunks must not be NULL");
        if (!oi) fail(DG_INVALID_INPUT, "intensity output must not be NULL");
        if ((flags & DG_ERRORS) && !os) fail(DG_INVALID_INPUT, "errors requested without an output");
        if ((flags & DG_AZIMUTHAL_STD) && !od)
            fail(DG_INVALID_INPUT, "azimuthal_std requested without an output");
        if ((flags & DG_AZIMUTHAL_STD) && plan->n_azimuthal != 0)
            fail(DG_UNSUPPORTED, "azimuthal_std is defined for 1D tables only");
        const int elem = dtype == DG_U16 ? 2 : 4;
        const int64_t npix = int64_t(plan->dim1) * plan->dim2;
        // every header first: a chunk that does not match the plan fails
        // before any device work
        std::vector<ChunkHead> heads(static_cast<size_t>(n_frames));
        for (int64_t f = 0; f < n_frames; ++f) {
            if (!chunks[f] || chunk_bytes[f] < 0)
                fail(DG_INVALID_INPUT, "frame " + std::to_string(f) + ": missing chunk");
            if (uint64_t(chunk_bytes[f]) > uint64_t(UINT32_MAX))
                fail(DG_INVALID_INPUT, "frame " + std::to_string(f) + ": chunk exceeds 4 GiB");
            heads[size_t(f)] = check_header(static_cast<const uint8_t *>(chunks[f]),
                                            chunk_bytes[f], f, npix, elem);
        }
        std::lock_guard<std::mutex> lock(plan->mu);
        int previous = -1;
        DG_CUDA(cudaGetDevice(&previous));
        struct Restore {
            int dev;
            ~Restore() {
                int now = -1;
                if (dev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != dev) cudaSetDevice(dev);
            }
        } restore{previous};
        if (previous != plan->device) DG_CUDA(cudaSetDevice(plan->device));

        const int64_t nb = plan->n_bins;
        const int nout = 1 + ((flags & DG_ERRORS) ? 1 : 0) + ((flags & DG_AZIMUTHAL_STD) ? 1 : 0);
        // Frames per batch: at most max_batch_frames and 64, and few enough
        // that element offsets fit 32 bits; compressed bytes of a batch fit
        // 32-bit offsets too.
        const int64_t tile = std::max<int64_t>(
            1, std::min<int64_t>({plan->max_batch_frames, int64_t(64), int64_t(UINT32_MAX) / npix}));
        struct Batch {
            int64_t f0 = 0, nf = 0;
            uint64_t comp = 0;
            uint32_t max_block = 0;
            size_t n_desc = 0;
            std::vector<size_t> desc_at;  // per frame: its first descriptor
            std::vector<BlockDesc> descs;
        };
        std::vector<Batch> batches;
        for (int64_t f = 0; f < n_frames;) {
            Batch bt;
            bt.f0 = f;
            while (f < n_frames && bt.nf < tile) {
                const uint64_t len = uint64_t(chunk_bytes[f]);
                if (bt.comp + len > uint64_t(UINT32_MAX)) break;
                bt.comp += len;
                bt.desc_at.push_back(bt.n_desc);
                bt.n_desc += heads[size_t(f)].n_desc;
                bt.max_block = std::max(bt.max_block, heads[size_t(f)].block);
                ++bt.nf;
                ++f;
            }
            batches.push_back(std::move(bt));
        }
        uint64_t comp_cap = 0;
        size_t desc_cap = 0;
        for (const Batch &bt : batches) {
            comp_cap = std::max(comp_cap, bt.comp);
            desc_cap = std::max(desc_cap, bt.n_desc);
        }
        const int64_t chunk = std::min<int64_t>(tile, n_frames);
        if (plan->stage_in.count < size_t(chunk * npix * elem)) {
            plan->stage_in.release();
            plan->stage_in.alloc(size_t(chunk * npix * elem));
        }
        if (plan->stage_out.count < size_t(chunk * nb * nout)) {
            plan->stage_out.release();
            plan->stage_out.alloc(size_t(chunk * nb * nout));
        }
        // Two slots of compressed bytes and of descriptors (256-byte aligned
        // starts and ends), and the error flag after the descriptors.
        const size_t comp_slot = (size_t(comp_cap) + 255) / 256 * 256;
        const size_t desc_slot = (desc_cap * sizeof(BlockDesc) + 255) / 256 * 256;
        const size_t n_slots = batches.size() > 1 ? 2 : 1;
        if (plan->stage_comp.count < n_slots * comp_slot) {
            plan->stage_comp.release();
            plan->stage_comp.alloc(n_slots * comp_slot);
        }
        if (plan->stage_desc.count < n_slots * desc_slot + 256) {
            plan->stage_desc.release();
            plan->stage_desc.alloc(n_slots * desc_slot + 256);
        }
        ensure_copy_pipeline(plan);
        cudaStream_t s = plan->stream, cs = plan->copy_stream;
        int *d_err = reinterpret_cast<int *>(plan->stage_desc.ptr + n_slots * desc_slot);
        DG_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), s));
        // the copy stream starts after everything already queued on the plan
        DG_CUDA(cudaEventRecord(plan->bs_decoded[0], s));
        DG_CUDA(cudaStreamWaitEvent(cs, plan->bs_decoded[0], 0));
        const int threads = int(std::min<unsigned>(8, std::max(1u, std::thread::hardware_concurrency())));

        auto copy_chunks = [&](size_t bi) {
            const size_t slot = bi % n_slots;
            const Batch &bt = batches[bi];
            // the slot's previous batch must have been decoded
            if (bi >= n_slots) DG_CUDA(cudaStreamWaitEvent(cs, plan->bs_decoded[slot], 0));
            unsigned char *dc = plan->stage_comp.ptr + slot * comp_slot;
            uint64_t at = 0;
            for (int64_t k = 0; k < bt.nf; ++k) {
                const int64_t f = bt.f0 + k;
                if (chunk_bytes[f])
                    DG_CUDA(cudaMemcpyAsync(dc + at, chunks[f], size_t(chunk_bytes[f]),
                                            cudaMemcpyHostToDevice, cs));
                at += uint64_t(chunk_bytes[f]);
            }
        };
        auto walk_and_copy_descs = [&](size_t bi) {
            const size_t slot = bi % n_slots;
            Batch &bt = batches[bi];
            bt.descs.resize(bt.n_desc);
            std::vector<uint64_t> base(static_cast<size_t>(bt.nf));
            for (int64_t k = 1; k < bt.nf; ++k)
                base[size_t(k)] = base[size_t(k - 1)] + uint64_t(chunk_bytes[bt.f0 + k - 1]);
            parallel_for(bt.nf, bt.n_desc > 4096 ? threads : 1, [&](int64_t k) {
                const int64_t f = bt.f0 + k;
                walk_blocks(static_cast<const uint8_t *>(chunks[f]), chunk_bytes[f], f, k,
                            base[size_t(k)], npix, elem, heads[size_t(f)],
                            bt.descs.data() + bt.desc_at[size_t(k)]);
            });
            if (bt.n_desc)
                DG_CUDA(cudaMemcpyAsync(plan->stage_desc.ptr + slot * desc_slot, bt.descs.data(),
                                        bt.n_desc * sizeof(BlockDesc), cudaMemcpyHostToDevice, cs));
            DG_CUDA(cudaEventRecord(plan->bs_copied[slot], cs));
        };
        copy_chunks(0);
        walk_and_copy_descs(0);
        for (size_t bi = 0; bi < batches.size(); ++bi) {
            const size_t slot = bi % n_slots;
            const Batch &bt = batches[bi];
            DG_CUDA(cudaStreamWaitEvent(s, plan->bs_copied[slot], 0));
            const uint32_t nblk = uint32_t(bt.n_desc);
            const uint32_t region = region_bytes(bt.max_block);
            const int warps = int(std::min<size_t>(4, kSmemPerSm / region));
            const size_t smem = size_t(warps) * region;
            const unsigned grid = (nblk + warps - 1) / warps;
            auto *bd = reinterpret_cast<const BlockDesc *>(plan->stage_desc.ptr + slot * desc_slot);
            const uint8_t *dc = plan->stage_comp.ptr + slot * comp_slot;
            if (nblk) {
                if (plan->gather.profile) record(plan->decode_events, s, true);
                ++plan->gather.launches;
                if (elem == 2) {
                    if (smem > plan->decode_smem[0]) {
                        DG_CUDA(cudaFuncSetAttribute(k_bslz4_decode<2>,
                                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     int(smem)));
                        plan->decode_smem[0] = smem;
                    }
                    k_bslz4_decode<2><<<grid, 32 * warps, smem, s>>>(
                        dc, bd, nblk, region, plan->stage_in.ptr, d_err);
                } else {
                    if (smem > plan->decode_smem[1]) {
                        DG_CUDA(cudaFuncSetAttribute(k_bslz4_decode<4>,
                                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     int(smem)));
                        plan->decode_smem[1] = smem;
                    }
                    k_bslz4_decode<4><<<grid, 32 * warps, smem, s>>>(
                        dc, bd, nblk, region, plan->stage_in.ptr, d_err);
                }
                DG_CUDA(cudaGetLastError());
                if (plan->gather.profile) record(plan->decode_events, s, false);
            }
            DG_CUDA(cudaEventRecord(plan->bs_decoded[slot], s));
            // the next batch's bytes travel while this batch is decoded
            if (bi + 1 < batches.size()) copy_chunks(bi + 1);
            const int64_t nf = bt.nf, f0 = bt.f0;
            double *di = plan->stage_out.ptr;
            double *ds = (flags & DG_ERRORS) ? di + nf * nb : nullptr;
            double *dd = (flags & DG_AZIMUTHAL_STD) ? di + nf * nb * (ds ? 2 : 1) : nullptr;
            run_gather(plan->gather, plan->stage_in.ptr, dtype, npix, nf, flags,
                       plan->method.precision, di, ds, dd, s);
            // the host walks the next batch's blocks while the device works
            if (bi + 1 < batches.size()) walk_and_copy_descs(bi + 1);
            DG_CUDA(cudaMemcpyAsync(oi + f0 * nb, di, size_t(nf * nb) * 8,
                                    cudaMemcpyDeviceToHost, s));
            if (ds)
                DG_CUDA(cudaMemcpyAsync(os + f0 * nb, ds, size_t(nf * nb) * 8,
                                        cudaMemcpyDeviceToHost, s));
            if (dd)
                DG_CUDA(cudaMemcpyAsync(od + f0 * nb, dd, size_t(nf * nb) * 8,
                                        cudaMemcpyDeviceToHost, s));
        }
        int herr = 0;
        DG_CUDA(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
        DG_CUDA(cudaStreamSynchronize(s));
        if (herr) fail(DG_INVALID_INPUT, "corrupt or truncated Bitshuffle/LZ4 compressed block");
        check_bin_tile_waits(plan->gather);
    });
    if (st != DG_OK && plan) {
        // leave nothing of this call in flight (queued copies read the
        // caller's chunks until they complete)
        if (plan->copy_stream) cudaStreamSynchronize(plan->copy_stream);
        if (plan->stream) cudaStreamSynchronize(plan->stream);
    }
    return st;
}

dg_status dg_plan_decode_time(dg_plan *plan, int32_t reset, double *ms, int64_t *launches) {
    using namespace dg;
    return guarded([&] {
        if (!plan) fail(DG_INVALID_INPUT, "plan must not be NULL");
        std::lock_guard<std::mutex> lock(plan->mu);
        EventPool &p = plan->decode_events;
        double total = 0.0;
        if (p.used) DG_CUDA(cudaEventSynchronize(p.events[p.used - 1].second));
        for (size_t i = 0; i < p.used; ++i) {
            float m = 0.f;
            DG_CUDA(cudaEventElapsedTime(&m, p.events[i].first, p.events[i].second));
            total += m;
        }
        if (ms) *ms = total;
        if (launches) *launches = int64_t(p.used);
        if (reset) p.used = 0;
    });
}

}  // extern "C"
