// TIFF movie reader (-InTiff): the role of TiffUtil/CLoadTiffHeader.cpp and
// TiffUtil/CLoadTiffImage.cpp, which read through libtiff.  Written from
// the TIFF 6.0 specification (and the BigTIFF extension): every image file
// directory is one raw frame; strips or tiles; no compression, LZW (with
// the TIFF "early change" code widths), Deflate (zlib) and PackBits;
// horizontal-differencing predictor.  Pixel types as CLoadTiffHeader::
// mReadMode (:121-148): 8 bits -> MRC mode 0, 16 bits -> 1 (signed sample
// format) or 6, 32-bit IEEE float -> 2.  Rows are stored bottom-up as
// CLoadTiffImage::mReadByStrip / mReadByTile write them (TIFF row r lands in
// frame row ny-1-r).  EER movies (-InEer) share the container parsing.
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mc3.h"

namespace {

struct Page {
  uint32_t nx = 0, ny = 0;
  int bits = 0, format = 1, compression = 1, predictor = 1, spp = 1;
  bool tiled = false;
  uint32_t rows_per_strip = 0, tile_w = 0, tile_h = 0;
  std::vector<uint64_t> offsets, counts;
};

struct File {
  bool big_endian = false;
  bool bigtiff = false;
  std::vector<Page> pages;
};

class Reader {
 public:
  explicit Reader(FILE* f, bool be) : f_(f), be_(be) {}
  bool read_at(uint64_t off, void* dst, size_t n) {
    if (fseeko(f_, (off_t)off, SEEK_SET) != 0) return false;
    return std::fread(dst, 1, n, f_) == n;
  }
  uint64_t uint(const uint8_t* p, int n) const {
    uint64_t v = 0;
    for (int i = 0; i < n; ++i) v |= (uint64_t)p[be_ ? n - 1 - i : i] << (8 * i);
    return v;
  }

 private:
  FILE* f_;
  bool be_;
};

int type_size(int t) {
  switch (t) {
    case 1: case 2: case 6: case 7: return 1;
    case 3: case 8: return 2;
    case 4: case 9: case 11: case 13: return 4;
    case 5: case 10: case 12: case 16: case 17: case 18: return 8;
    default: return 0;
  }
}

// Values of one directory entry as unsigned integers (SHORT, LONG, LONG8).
bool entry_values(Reader& r, bool big, const uint8_t* e, std::vector<uint64_t>& out) {
  const int type = (int)r.uint(e + 2, 2);
  const uint64_t count = big ? r.uint(e + 4, 8) : r.uint(e + 4, 4);
  const int ts = type_size(type);
  if (!ts || count > (1u << 26)) return false;
  const size_t bytes = (size_t)ts * count;
  const int inline_cap = big ? 8 : 4;
  std::vector<uint8_t> buf(bytes);
  const uint8_t* src = e + (big ? 12 : 8);
  if (bytes <= (size_t)inline_cap) {
    std::memcpy(buf.data(), src, bytes);
  } else {
    const uint64_t off = big ? r.uint(src, 8) : r.uint(src, 4);
    if (!r.read_at(off, buf.data(), bytes)) return false;
  }
  out.resize(count);
  for (uint64_t i = 0; i < count; ++i) {
    if (type == 5) {  // RATIONAL: numerator only (not used for sizes)
      out[i] = r.uint(buf.data() + 8 * i, 4);
    } else {
      out[i] = r.uint(buf.data() + (size_t)ts * i, ts > 8 ? 8 : ts);
    }
  }
  return true;
}

bool parse(const char* path, File& tf) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  uint8_t h[16];
  bool ok = std::fread(h, 1, 16, f) >= 8;
  if (ok) {
    if (h[0] == 'I' && h[1] == 'I') tf.big_endian = false;
    else if (h[0] == 'M' && h[1] == 'M') tf.big_endian = true;
    else ok = false;
  }
  Reader r(f, tf.big_endian);
  uint64_t ifd = 0;
  if (ok) {
    const uint64_t magic = r.uint(h + 2, 2);
    if (magic == 42) {
      ifd = r.uint(h + 4, 4);
    } else if (magic == 43) {
      tf.bigtiff = true;
      ifd = r.uint(h + 8, 8);
    } else {
      ok = false;
    }
  }
  const bool big = tf.bigtiff;
  std::vector<uint64_t> seen;
  while (ok && ifd != 0) {
    if (std::find(seen.begin(), seen.end(), ifd) != seen.end()) break;  // a loop
    seen.push_back(ifd);
    uint8_t cb[8];
    if (!r.read_at(ifd, cb, big ? 8 : 2)) { ok = false; break; }
    const uint64_t n = r.uint(cb, big ? 8 : 2);
    const int esz = big ? 20 : 12;
    if (n > 4096) { ok = false; break; }
    std::vector<uint8_t> ents((size_t)n * esz + (big ? 8 : 4));
    if (!r.read_at(ifd + (big ? 8 : 2), ents.data(), ents.size())) { ok = false; break; }
    Page pg;
    for (uint64_t i = 0; i < n && ok; ++i) {
      const uint8_t* e = ents.data() + i * esz;
      const int tag = (int)r.uint(e, 2);
      std::vector<uint64_t> v;
      switch (tag) {
        case 256: case 257: case 258: case 259: case 273: case 277: case 278: case 279:
        case 317: case 322: case 323: case 324: case 325: case 339:
          if (!entry_values(r, big, e, v) || v.empty()) { ok = false; break; }
          if (tag == 256) pg.nx = (uint32_t)v[0];
          else if (tag == 257) pg.ny = (uint32_t)v[0];
          else if (tag == 258) pg.bits = (int)v[0];
          else if (tag == 259) pg.compression = (int)v[0];
          else if (tag == 277) pg.spp = (int)v[0];
          else if (tag == 278) pg.rows_per_strip = (uint32_t)v[0];
          else if (tag == 317) pg.predictor = (int)v[0];
          else if (tag == 322) { pg.tile_w = (uint32_t)v[0]; pg.tiled = true; }
          else if (tag == 323) pg.tile_h = (uint32_t)v[0];
          else if (tag == 339) pg.format = (int)v[0];
          else if (tag == 273 || tag == 324) pg.offsets = v;
          else pg.counts = v;
          break;
        default: break;
      }
    }
    if (!ok) break;
    if (pg.rows_per_strip == 0 || pg.rows_per_strip > pg.ny) pg.rows_per_strip = pg.ny;
    tf.pages.push_back(pg);
    const uint8_t* nxt = ents.data() + n * esz;
    ifd = r.uint(nxt, big ? 8 : 4);
  }
  std::fclose(f);
  return ok && !tf.pages.empty();
}

// CLoadTiffHeader::mReadMode (TiffUtil/CLoadTiffHeader.cpp:121-148).
int page_mode(const Page& p) {
  if (p.spp != 1) return -1;
  if (p.bits == 8) return 0;
  if (p.bits == 16) return p.format == 2 ? 1 : 6;
  if (p.format == 3 && p.bits == 32) return 2;
  return -1;
}

// ---- decoders: each fills out[0..cap) from in[0..n) ----
// TIFF 6.0 section 13 LZW: MSB-first codes, Clear 256, EOI 257, widths 9..12
// bits, switching one code early (when the next free code + 1 reaches 2^w).
bool lzw_decode(const uint8_t* in, size_t n, uint8_t* out, size_t cap) {
  struct Ent { int prev; uint8_t first, last; int len; };
  std::vector<Ent> tab(4096);
  for (int i = 0; i < 256; ++i) tab[i] = Ent{-1, (uint8_t)i, (uint8_t)i, 1};
  int next = 258, width = 9, old = -1;
  size_t o = 0, ip = 0;
  uint64_t bitbuf = 0;
  int bits = 0;
  auto emit = [&](int code) {
    const int len = tab[code].len;
    const size_t room = cap - o;
    int c = code;
    // write back to front; drop what does not fit (last strip padding)
    for (int k = len - 1; k >= 0; --k) {
      if ((size_t)k < room) out[o + k] = tab[c].last;
      c = tab[c].prev;
    }
    o += std::min((size_t)len, room);
  };
  while (o < cap) {
    while (bits < width && ip < n) {
      bitbuf = (bitbuf << 8) | in[ip++];
      bits += 8;
    }
    if (bits < width) break;
    const int code = (int)((bitbuf >> (bits - width)) & ((1u << width) - 1));
    bits -= width;
    if (code == 257) break;
    if (code == 256) {
      next = 258;
      width = 9;
      old = -1;
      continue;
    }
    if (old < 0) {
      if (code > 255) return false;
      emit(code);
      old = code;
      continue;
    }
    uint8_t first;
    if (code < next) first = tab[code].first;
    else if (code == next) first = tab[old].first;  // the KwKwK case
    else return false;
    if (next < 4096) {
      tab[next] = Ent{old, tab[old].first, first, tab[old].len + 1};
      ++next;
    }
    emit(code);
    old = code;
    if (next + 1 >= (1 << width) && width < 12) ++width;
  }
  return o == cap;
}

// PackBits (TIFF 6.0 section 9).
bool packbits_decode(const uint8_t* in, size_t n, uint8_t* out, size_t cap) {
  size_t ip = 0, o = 0;
  while (ip < n && o < cap) {
    const int8_t h = (int8_t)in[ip++];
    if (h >= 0) {
      const size_t c = (size_t)h + 1;
      if (ip + c > n) return false;
      const size_t w = std::min(c, cap - o);
      std::memcpy(out + o, in + ip, w);
      ip += c;
      o += w;
    } else if (h != -128) {
      if (ip >= n) return false;
      const size_t c = (size_t)(1 - h);
      const size_t w = std::min(c, cap - o);
      std::memset(out + o, in[ip++], w);
      o += w;
    }
  }
  return o == cap;
}

bool inflate_decode(const uint8_t* in, size_t n, uint8_t* out, size_t cap) {
  z_stream zs;
  std::memset(&zs, 0, sizeof(zs));
  if (inflateInit(&zs) != Z_OK) return false;
  zs.next_in = const_cast<Bytef*>(in);
  zs.avail_in = (uInt)n;
  zs.next_out = out;
  zs.avail_out = (uInt)cap;
  const int rc = inflate(&zs, Z_FINISH);
  const size_t got = cap - zs.avail_out;
  inflateEnd(&zs);
  return (rc == Z_STREAM_END || rc == Z_OK || rc == Z_BUF_ERROR) && got == cap;
}

// One strip or tile: `rows` rows of `w` pixels of `bpp` bytes, decoded and
// un-predicted into dst (row pitch w*bpp).
bool decode_block(const Page& pg, const uint8_t* in, size_t n, uint8_t* dst, uint32_t w,
                  uint32_t rows, int bpp, bool be) {
  const size_t cap = (size_t)w * rows * bpp;
  bool ok = false;
  switch (pg.compression) {
    case 1:
      ok = n >= cap;
      if (ok) std::memcpy(dst, in, cap);
      break;
    case 5: ok = lzw_decode(in, n, dst, cap); break;
    case 8: case 32946: ok = inflate_decode(in, n, dst, cap); break;
    case 32773: ok = packbits_decode(in, n, dst, cap); break;
    default: return false;
  }
  if (!ok) return false;
  // multi-byte samples to host (little-endian) order
  if (be && bpp > 1)
    for (size_t i = 0; i < cap; i += bpp) std::reverse(dst + i, dst + i + bpp);
  if (pg.predictor == 2) {  // horizontal differencing, integer samples
    for (uint32_t r = 0; r < rows; ++r) {
      uint8_t* row = dst + (size_t)r * w * bpp;
      if (bpp == 1) {
        for (uint32_t x = 1; x < w; ++x) row[x] = (uint8_t)(row[x] + row[x - 1]);
      } else if (bpp == 2) {
        uint16_t* p = reinterpret_cast<uint16_t*>(row);
        for (uint32_t x = 1; x < w; ++x) p[x] = (uint16_t)(p[x] + p[x - 1]);
      } else {
        return false;
      }
    }
  } else if (pg.predictor != 1) {
    return false;
  }
  return true;
}

// Frame `z` into dst (ny rows of nx pixels, bottom-up).
bool read_page(FILE* f, const Page& pg, bool be, uint8_t* dst) {
  const int mode = page_mode(pg);
  const int bpp = mode == 0 ? 1 : (mode == 2 ? 4 : 2);
  const uint32_t nx = pg.nx, ny = pg.ny;
  const size_t row_bytes = (size_t)nx * bpp;
  std::vector<uint8_t> comp, blk;
  auto fetch = [&](size_t i) -> bool {
    if (i >= pg.offsets.size() || i >= pg.counts.size()) return false;
    comp.resize(pg.counts[i]);
    if (fseeko(f, (off_t)pg.offsets[i], SEEK_SET) != 0) return false;
    return std::fread(comp.data(), 1, comp.size(), f) == comp.size();
  };
  if (!pg.tiled) {  // CLoadTiffImage::mReadByStrip (:70-110)
    const uint32_t rps = pg.rows_per_strip;
    const size_t nstrips = (ny + rps - 1) / rps;
    for (size_t i = 0; i < nstrips; ++i) {
      const uint32_t r0 = (uint32_t)i * rps;
      const uint32_t rows = std::min(rps, ny - r0);
      if (!fetch(i)) return false;
      blk.resize((size_t)rows * row_bytes);
      if (!decode_block(pg, comp.data(), comp.size(), blk.data(), nx, rows, bpp, be)) return false;
      for (uint32_t r = 0; r < rows; ++r)
        std::memcpy(dst + (size_t)(ny - 1 - (r0 + r)) * row_bytes, blk.data() + r * row_bytes,
                    row_bytes);
    }
    return true;
  }
  // CLoadTiffImage::mReadByTile (:112-160): whole tiles are decoded, their
  // parts inside the image copied bottom-up (the reference's pointer
  // arithmetic there is in bytes of 8-bit samples; wider samples are placed
  // by pixel here)
  const uint32_t tw = pg.tile_w, th = pg.tile_h;
  if (!tw || !th) return false;
  const uint32_t ntx = (nx + tw - 1) / tw, nty = (ny + th - 1) / th;
  blk.resize((size_t)tw * th * bpp);
  for (uint32_t ty = 0; ty < nty; ++ty)
    for (uint32_t tx = 0; tx < ntx; ++tx) {
      if (!fetch((size_t)ty * ntx + tx)) return false;
      if (!decode_block(pg, comp.data(), comp.size(), blk.data(), tw, th, bpp, be)) return false;
      const uint32_t x0 = tx * tw, w = std::min(tw, nx - x0);
      for (uint32_t r = 0; r < th && ty * th + r < ny; ++r) {
        const uint32_t row = ty * th + r;
        std::memcpy(dst + (size_t)(ny - 1 - row) * row_bytes + (size_t)x0 * bpp,
                    blk.data() + (size_t)r * tw * bpp, (size_t)w * bpp);
      }
    }
  return true;
}

// ---- EER (electron-event representation) frames --------------------------
// One TIFF directory per EER frame, its strips concatenated
// (EerUtil/CLoadEerFrames.cpp:77-95); compression 65001 = 7-bit run lengths,
// 65000 = 8-bit run lengths, each followed by a 4-bit sub-pixel code
// (EerUtil/CLoadEerHeader.cpp:22-51).
struct EerDecoder {
  int cam_w = 0, cam_h = 0, bits = 0, sampling = 1;
  int frm_w = 0;
  // sub-pixel bit selection of CDecodeEerFrame::Setup (EerUtil/CDecodeEerFrame.cpp:17-41)
  int sh0 = 0, and0 = 0, sh1 = 0, and1 = 0, sh2 = 0;
  bool setup(int w, int h, int b, int smp) {
    cam_w = w;
    cam_h = h;
    bits = b;
    sampling = smp;
    const int fact = smp == 2 ? 2 : (smp == 3 ? 4 : 1);
    if (smp == 2) { sh0 = 1; and0 = 2; sh1 = 1; and1 = 8; sh2 = 3; }
    if (smp == 3) { sh0 = 2; and0 = 3; sh1 = 0; and1 = 12; sh2 = 2; }
    frm_w = w * fact;
    // the super-resolution position arithmetic assumes 4096-pixel rows
    return smp == 1 || w == 4096;
  }
  // CDecodeEerFrame::mFindElectron (:167-175)
  void electron(uint32_t n, unsigned s, uint8_t* frm) const {
    const uint32_t x = ((n & 4095u) << sh0) | ((s & and0) >> sh1);
    const uint32_t y = ((n >> 12) << sh0) | ((s & and1) >> sh2);
    frm[(size_t)y * frm_w + x] += 1;
  }
  // Adds the electrons of one EER frame to frm (8-bit counts).
  void decode(const uint8_t* d, size_t n, uint8_t* frm) const {
    const uint32_t cam = (uint32_t)cam_w * cam_h;
    uint32_t pix = 0;
    if (bits == 7) {  // mDo7BitsCounted / mDo7BitsSuperRes (:55-117)
      uint64_t pos = 0;
      const uint64_t end = (uint64_t)n * 8;
      auto get = [&](int nb) {
        unsigned v = 0;
        for (int k = 0; k < nb; ++k, ++pos)
          if (pos < end) v |= ((d[pos >> 3] >> (pos & 7)) & 1u) << k;
        return v;
      };
      while (pos < end) {
        const unsigned run = get(7);
        pix += run;
        if (pix >= cam) break;
        if (run == 127) continue;
        const unsigned sub = get(4) ^ 0x0Au;
        if (sampling == 1) {
          frm[(size_t)(pix / frm_w) * frm_w + pix % frm_w] += 1;
        } else {
          electron(pix, sub, frm);
        }
        pix += 1;
      }
      return;
    }
    // 8 bits: three bytes carry two (run, sub-pixel) codes (:119-165)
    for (size_t p = 0; p + 2 < n; p += 3) {
      const unsigned p1 = d[p];
      unsigned s1 = d[p + 1] & 0x0Au;
      pix += p1;
      if (pix >= cam) break;
      if (p1 < 255) {
        if (sampling == 1) frm[(size_t)(pix / frm_w) * frm_w + pix % frm_w] += 1;
        else electron(pix, s1, frm);
        pix += 1;
      }
      unsigned p2, s2;
      if (sampling == 1) {
        p2 = ((d[p + 1] >> 4) | (d[p + 2] << 4)) & 0xFFu;
        s2 = 0;
      } else {
        // the reference's super-resolution branch reads its third byte
        // from offset 0 of the frame (uiPos2 is never advanced, :150-156)
        p2 = ((d[p + 1] >> 4) | d[0]) & 0xFFu;
        s2 = ((unsigned)(d[0] >> 4)) ^ 0x0Au;
      }
      pix += p2;
      if (pix >= cam) break;
      if (p2 < 255) {
        if (sampling == 1) frm[(size_t)(pix / frm_w) * frm_w + pix % frm_w] += 1;
        else electron(pix, s2, frm);
        pix += 1;
      }
    }
  }
};

int eer_bits(const Page& p) {
  if (p.compression == 65001) return 7;
  if (p.compression == 65000) return 8;
  return -1;  // 65002 is not decoded by the reference either (CLoadEerHeader.cpp:34-39)
}

}  // namespace

extern "C" {

int mc3_eer_info(const char* path, int* cam_x, int* cam_y, int* n_frames, int* bits) {
  if (!path) return MC3_EINVAL;
  File tf;
  if (!parse(path, tf)) return MC3_EIO;
  const Page& p0 = tf.pages[0];
  const int b = eer_bits(p0);
  if (b < 0 || p0.nx == 0 || p0.ny == 0) return MC3_EUNSUPPORTED;
  if (cam_x) *cam_x = (int)p0.nx;
  if (cam_y) *cam_y = (int)p0.ny;
  if (n_frames) *n_frames = (int)tf.pages.size();
  if (bits) *bits = b;
  return MC3_OK;
}

int mc3_eer_render(const char* path, int sampling, int n_out, const int* start, const int* size,
                   unsigned char* dst, int threads) {
  if (!path || !dst || n_out < 1 || !start || !size) return MC3_EINVAL;
  if (sampling < 1 || sampling > 3) return MC3_EINVAL;
  File tf;
  if (!parse(path, tf)) return MC3_EIO;
  const Page& p0 = tf.pages[0];
  EerDecoder dec;
  const int b = eer_bits(p0);
  if (b < 0 || !dec.setup((int)p0.nx, (int)p0.ny, b, sampling)) return MC3_EUNSUPPORTED;
  const int fact = sampling == 2 ? 2 : (sampling == 3 ? 4 : 1);
  const size_t frame = (size_t)p0.nx * fact * p0.ny * fact;
  for (int i = 0; i < n_out; ++i)
    if (start[i] < 0 || size[i] < 1 || start[i] + size[i] > (int)tf.pages.size()) return MC3_EINVAL;
  // CRenderMrcStack::mRender / mRenderInt (EerUtil/CRenderMrcStack.cpp:30-95):
  // rendered frame i = the electrons of EER frames start[i] .. start[i]+size[i]-1
  int nt = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
  nt = std::max(1, std::min(nt, n_out));
  std::atomic<int> next{0};
  std::atomic<int> status{MC3_OK};
  auto work = [&]() {
    FILE* f = std::fopen(path, "rb");
    if (!f) {
      status = MC3_EIO;
      return;
    }
    std::vector<uint8_t> buf;
    for (;;) {
      const int i = next.fetch_add(1);
      if (i >= n_out || status != MC3_OK) break;
      uint8_t* frm = dst + frame * i;
      std::memset(frm, 0, frame);
      for (int k = 0; k < size[i] && status == MC3_OK; ++k) {
        const Page& pg = tf.pages[start[i] + k];
        if (pg.nx != p0.nx || pg.ny != p0.ny || eer_bits(pg) != b) {
          status = MC3_EUNSUPPORTED;
          break;
        }
        size_t tot = 0;
        for (size_t s = 0; s < pg.offsets.size() && s < pg.counts.size(); ++s) tot += pg.counts[s];
        buf.assign(tot + 8, 0);  // zero tail: bit reads past the data see zeros
        size_t o = 0;
        for (size_t s = 0; s < pg.offsets.size() && s < pg.counts.size(); ++s) {
          if (fseeko(f, (off_t)pg.offsets[s], SEEK_SET) != 0 ||
              std::fread(buf.data() + o, 1, pg.counts[s], f) != pg.counts[s]) {
            status = MC3_EIO;
            break;
          }
          o += pg.counts[s];
        }
        if (status == MC3_OK) dec.decode(buf.data(), tot, frm);
      }
    }
    std::fclose(f);
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t) pool.emplace_back(work);
  for (auto& t : pool) t.join();
  return status;
}

int mc3_tiff_info(const char* path, int* nx, int* ny, int* nz, int* mode) {
  if (!path) return MC3_EINVAL;
  File tf;
  if (!parse(path, tf)) return MC3_EIO;
  const Page& p0 = tf.pages[0];
  const int m = page_mode(p0);
  if (m < 0) return MC3_EUNSUPPORTED;
  for (const Page& p : tf.pages)
    if (p.nx != p0.nx || p.ny != p0.ny || page_mode(p) != m) return MC3_EUNSUPPORTED;
  if (nx) *nx = (int)p0.nx;
  if (ny) *ny = (int)p0.ny;
  if (nz) *nz = (int)tf.pages.size();
  if (mode) *mode = m;
  return MC3_OK;
}

int mc3_tiff_read(const char* path, int z0, int nz, void* dst, int threads) {
  if (!path || !dst || z0 < 0 || nz < 1) return MC3_EINVAL;
  File tf;
  if (!parse(path, tf)) return MC3_EIO;
  if (z0 + nz > (int)tf.pages.size()) return MC3_EINVAL;
  const Page& p0 = tf.pages[0];
  const int m = page_mode(p0);
  if (m < 0) return MC3_EUNSUPPORTED;
  const size_t frame = (size_t)p0.nx * p0.ny * (m == 0 ? 1 : (m == 2 ? 4 : 2));
  // CLoadTiffStack reads frames on several threads (TiffUtil/CLoadTiffStack.cpp:104-118)
  int nt = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
  nt = std::max(1, std::min(nt, nz));
  std::atomic<int> next{0};
  std::atomic<int> status{MC3_OK};
  auto work = [&]() {
    FILE* f = std::fopen(path, "rb");
    if (!f) {
      status = MC3_EIO;
      return;
    }
    for (;;) {
      const int i = next.fetch_add(1);
      if (i >= nz || status != MC3_OK) break;
      const Page& pg = tf.pages[z0 + i];
      if (pg.nx != p0.nx || pg.ny != p0.ny || page_mode(pg) != m) {
        status = MC3_EUNSUPPORTED;
        break;
      }
      if (!read_page(f, pg, tf.big_endian, static_cast<uint8_t*>(dst) + frame * i)) {
        status = MC3_EIO;
        break;
      }
    }
    std::fclose(f);
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t) pool.emplace_back(work);
  for (auto& t : pool) t.join();
  return status;
}

}  // extern "C"
