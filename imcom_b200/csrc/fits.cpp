// fits.cpp -- FITS image files without CFITSIO (host code).
//
// The reference reads its input images, coordinate maps and PSFs, and reads
// and writes its A/B/Q/L/P/T cache and U/S/K maps, through CFITSIO
// (imcom_io.f90:338-494: imcom_sizefits, imcom_readfits, imcom_writefits,
// imcom_writefitscube).  These functions do the same for the primary HDU of
// a FITS file (the FITS Standard 4.0: 2880-byte blocks of 80-character
// header cards, big-endian data), so a driver that gets its arrays from the
// C-ABI needs no CFITSIO for them.
//
//   imcom_fits_size   NAXIS1, NAXIS2 and BITPIX of the primary image.
//   imcom_fits_read   the image as doubles: every BITPIX (8, 16, 32, 64, -32,
//                     -64) with BSCALE / BZERO applied; NaN pixels of
//                     floating-point images and BLANK pixels of integer images
//                     become -666 (the null value imcom_readfits passes to
//                     FTGPVD); sizes must match the caller's, as there.
//   imcom_fits_write  a BITPIX -64 image, replacing an existing file.
//   imcom_fits_write_cube  the same with three axes.
//
// Errors return IMCOM_ERR_FITS with a message in imcom_fits_last_error()
// (per host thread); bad arguments return -k.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/imcom_gpu.h"

namespace {

constexpr size_t kBlock = 2880, kCard = 80;
constexpr double kNull = -666.0;  // imcom_readfits' null value (imcom_io.f90:366)

thread_local std::string g_fits_err;

int fail(const char* fmt, ...) __attribute__((format(printf, 1, 2)));
int fail(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_fits_err = buf;
  return IMCOM_ERR_FITS;
}

struct Header {
  int bitpix = 0, naxis = 0;
  long long naxes[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double bscale = 1.0, bzero = 0.0;
  bool has_blank = false;
  long long blank = 0;
  size_t data_offset = 0;
};

std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(' '), b = s.find_last_not_of(' ');
  return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

// Value field of a card (columns 11-80) up to a comment slash outside quotes.
std::string card_value(const char* card) {
  std::string v(card + 10, kCard - 10);
  bool quoted = false;
  for (size_t i = 0; i < v.size(); ++i) {
    if (v[i] == '\'') quoted = !quoted;
    if (v[i] == '/' && !quoted) {
      v.resize(i);
      break;
    }
  }
  return trim(v);
}

bool parse_int(const std::string& v, long long* out) {
  if (v.empty()) return false;
  char* end = nullptr;
  errno = 0;
  long long x = strtoll(v.c_str(), &end, 10);
  if (errno || *end) return false;
  *out = x;
  return true;
}

bool parse_real(const std::string& v, double* out) {
  if (v.empty()) return false;
  std::string t = v;
  for (char& c : t)
    if (c == 'D' || c == 'd') c = 'E';  // FITS allows a D exponent
  char* end = nullptr;
  errno = 0;
  double x = strtod(t.c_str(), &end);
  if (errno || *end) return false;
  *out = x;
  return true;
}

int read_header(FILE* f, const char* path, Header* h) {
  char card[kCard];
  bool simple = false, end = false;
  size_t ncard = 0;
  while (!end) {
    if (fread(card, 1, kCard, f) != kCard)
      return fail("%s: no END card in the primary header", path);
    const std::string key = trim(std::string(card, 8));
    const bool valued = card[8] == '=' && card[9] == ' ';
    if (ncard == 0) {
      if (key != "SIMPLE" || !valued || card_value(card) != "T")
        return fail("%s: not a FITS file (first card is not SIMPLE = T)", path);
      simple = true;
    } else if (key == "END") {
      end = true;
    } else if (valued) {
      const std::string v = card_value(card);
      long long iv = 0;
      double dv = 0.0;
      if (key == "BITPIX") {
        if (!parse_int(v, &iv)) return fail("%s: bad BITPIX", path);
        h->bitpix = (int)iv;
      } else if (key == "NAXIS") {
        if (!parse_int(v, &iv) || iv < 0 || iv > 8) return fail("%s: bad NAXIS", path);
        h->naxis = (int)iv;
      } else if (key.size() > 5 && key.compare(0, 5, "NAXIS") == 0) {
        long long ax = 0;
        if (parse_int(key.substr(5), &ax) && ax >= 1 && ax <= 8) {
          if (!parse_int(v, &iv) || iv < 0) return fail("%s: bad %s", path, key.c_str());
          h->naxes[ax - 1] = iv;
        }
      } else if (key == "BSCALE") {
        if (!parse_real(v, &dv)) return fail("%s: bad BSCALE", path);
        h->bscale = dv;
      } else if (key == "BZERO") {
        if (!parse_real(v, &dv)) return fail("%s: bad BZERO", path);
        h->bzero = dv;
      } else if (key == "BLANK") {
        if (!parse_int(v, &iv)) return fail("%s: bad BLANK", path);
        h->blank = iv;
        h->has_blank = true;
      }
    }
    ++ncard;
  }
  if (!simple) return fail("%s: not a FITS file", path);
  switch (h->bitpix) {
    case 8: case 16: case 32: case 64: case -32: case -64: break;
    default: return fail("%s: BITPIX %d is not a FITS data type", path, h->bitpix);
  }
  if (h->naxis < 1) return fail("%s: the primary HDU holds no image (NAXIS = 0)", path);
  const size_t header_bytes = ncard * kCard;
  h->data_offset = (header_bytes + kBlock - 1) / kBlock * kBlock;
  return 0;
}

int open_header(const char* path, FILE** fp, Header* h) {
  FILE* f = fopen(path, "rb");
  if (!f) return fail("%s: cannot open (%s)", path, strerror(errno));
  const int st = read_header(f, path, h);
  if (st) {
    fclose(f);
    return st;
  }
  *fp = f;
  return 0;
}

// Values per read or write chunk (1 MiB of doubles).
constexpr size_t kChunk = 131072;

inline uint8_t swap_bytes(uint8_t u) { return u; }
inline uint16_t swap_bytes(uint16_t u) { return __builtin_bswap16(u); }
inline uint32_t swap_bytes(uint32_t u) { return __builtin_bswap32(u); }
inline uint64_t swap_bytes(uint64_t u) { return __builtin_bswap64(u); }

// nb stored values of type T (big-endian, at src) to doubles at out, with
// no branch inside the loop (the null test is a select, the scaling a
// template flag), so the compiler vectorises the swap.  kInPlace (8-byte
// types only) reads each value from its own slot of out, which the
// compiler can see is the slot it then writes.
template <class T, class U, bool kScaled, bool kInPlace>
inline void decode_values(const unsigned char* src, size_t nb, const Header& h, double* out) {
  static_assert(sizeof(T) == sizeof(U), "stored type and its bit pattern differ in width");
  static_assert(!kInPlace || sizeof(T) == sizeof(double), "in place needs 8-byte values");
  const double bscale = h.bscale, bzero = h.bzero;
  const bool has_blank = h.has_blank;
  const T blank = (T)h.blank;
  // a BLANK outside the stored type's range never matches
  const bool blank_fits = (long long)blank == h.blank;
  for (size_t i = 0; i < nb; ++i) {
    U u;
    if constexpr (kInPlace)
      memcpy(&u, out + i, sizeof(U));
    else
      memcpy(&u, src + sizeof(U) * i, sizeof(U));
    u = swap_bytes(u);
    T x;
    memcpy(&x, &u, sizeof(T));
    bool null;
    if constexpr (std::is_floating_point<T>::value)
      null = x != x;
    else
      null = has_blank & blank_fits & (x == blank);
    double v = (double)x;
    if constexpr (kScaled) v = bzero + bscale * v;
    out[i] = null ? kNull : v;
  }
}

template <class T, class U>
inline void decode_typed(const unsigned char* src, size_t nb, const Header& h, bool scaled,
                         double* out) {
  if constexpr (sizeof(T) == sizeof(double)) {
    if (static_cast<const void*>(src) == static_cast<const void*>(out)) {
      if (scaled)
        decode_values<T, U, true, true>(src, nb, h, out);
      else
        decode_values<T, U, false, true>(src, nb, h, out);
      return;
    }
  }
  if (scaled)
    decode_values<T, U, true, false>(src, nb, h, out);
  else
    decode_values<T, U, false, false>(src, nb, h, out);
}

// Stored values of the header's BITPIX to doubles.  Built once per
// instruction set (AVX2 byte shuffles where the host has them, baseline
// x86-64 otherwise) and chosen when the library loads.
__attribute__((target_clones("avx2", "default")))
void decode_chunk(const unsigned char* src, size_t nb, const Header& h, bool scaled,
                  double* out) {
  switch (h.bitpix) {
    case -64: decode_typed<double, uint64_t>(src, nb, h, scaled, out); break;
    case -32: decode_typed<float, uint32_t>(src, nb, h, scaled, out); break;
    case 8: decode_typed<uint8_t, uint8_t>(src, nb, h, scaled, out); break;
    case 16: decode_typed<int16_t, uint16_t>(src, nb, h, scaled, out); break;
    case 32: decode_typed<int32_t, uint32_t>(src, nb, h, scaled, out); break;
    default: decode_typed<int64_t, uint64_t>(src, nb, h, scaled, out); break;
  }
}

__attribute__((target_clones("avx2", "default")))
void encode_chunk(const double* in, size_t nb, unsigned char* dst) {
  for (size_t i = 0; i < nb; ++i) {
    uint64_t u;
    memcpy(&u, in + i, 8);
    u = swap_bytes(u);
    memcpy(dst + 8 * i, &u, 8);
  }
}

// One header card "KEY     = value" with the value right-justified to
// column 30 (the fixed format) and a short comment.
void put_card(std::string* hdr, const char* key, const std::string& value, const char* comment) {
  char card[kCard + 1];
  snprintf(card, sizeof card, "%-8.8s= %20s / %-47.47s", key, value.c_str(), comment);
  hdr->append(card, kCard);
}

int write_image(const char* path, int naxis, const long long* naxes, const double* data) {
  if (!path || !*path) return -1;
  size_t count = 1;
  for (int a = 0; a < naxis; ++a) count *= (size_t)naxes[a];
  std::string hdr;
  put_card(&hdr, "SIMPLE", "T", "conforms to the FITS Standard");
  put_card(&hdr, "BITPIX", "-64", "IEEE double precision");
  put_card(&hdr, "NAXIS", std::to_string(naxis), "number of axes");
  static const char* names[3] = {"NAXIS1", "NAXIS2", "NAXIS3"};
  for (int a = 0; a < naxis; ++a)
    put_card(&hdr, names[a], std::to_string(naxes[a]), "length of the axis");
  put_card(&hdr, "EXTEND", "T", "extensions may follow");
  {
    std::string end = "END";
    end.resize(kCard, ' ');
    hdr += end;
  }
  hdr.resize((hdr.size() + kBlock - 1) / kBlock * kBlock, ' ');
  // the reference deletes an existing file before writing (imcom_io.f90:426-432)
  if (remove(path) != 0 && errno != ENOENT)
    return fail("%s: cannot replace the existing file (%s)", path, strerror(errno));
  FILE* f = fopen(path, "wb");
  if (!f) return fail("%s: cannot create (%s)", path, strerror(errno));
  bool ok = fwrite(hdr.data(), 1, hdr.size(), f) == hdr.size();
  std::vector<unsigned char> buf(8 * std::min(kChunk, std::max(count, (size_t)1)));
  for (size_t i0 = 0; ok && i0 < count; i0 += kChunk) {
    const size_t nb = std::min(kChunk, count - i0);
    encode_chunk(data + i0, nb, buf.data());
    ok = fwrite(buf.data(), 1, 8 * nb, f) == 8 * nb;
  }
  const size_t data_bytes = 8 * count;
  const size_t pad = (kBlock - data_bytes % kBlock) % kBlock;
  if (ok && pad) {
    std::vector<unsigned char> zeros(pad, 0);
    ok = fwrite(zeros.data(), 1, pad, f) == pad;
  }
  if (fclose(f) != 0) ok = false;
  if (!ok) return fail("%s: write failed", path);
  return 0;
}

}  // namespace

extern "C" const char* imcom_fits_last_error(void) { return g_fits_err.c_str(); }

extern "C" int imcom_fits_size(const char* path, int* naxis1, int* naxis2, int* bitpix) {
  if (!path) return -1;
  if (!naxis1) return -2;
  if (!naxis2) return -3;
  if (!bitpix) return -4;
  FILE* f = nullptr;
  Header h;
  const int st = open_header(path, &f, &h);
  if (st) return st;
  fclose(f);
  *naxis1 = (int)h.naxes[0];
  *naxis2 = h.naxis >= 2 ? (int)h.naxes[1] : 1;
  *bitpix = h.bitpix;
  return 0;
}

extern "C" int imcom_fits_read(const char* path, int naxis1, int naxis2, double* image) {
  if (!path) return -1;
  if (naxis1 < 0) return -2;
  if (naxis2 < 0) return -3;
  if (!image && (long long)naxis1 * naxis2 > 0) return -4;
  FILE* f = nullptr;
  Header h;
  int st = open_header(path, &f, &h);
  if (st) return st;
  long long count = 1;
  for (int a = 0; a < h.naxis; ++a) count *= h.naxes[a];
  const long long n2 = h.naxis >= 2 ? h.naxes[1] : 1;
  if (h.naxes[0] != naxis1) {
    fclose(f);
    return fail("%s: NAXIS1 is %lld, not the %d asked for", path, h.naxes[0], naxis1);
  }
  if (n2 != naxis2 || count != (long long)naxis1 * naxis2) {
    fclose(f);
    return fail("%s: the image holds %lld x %lld values, not %d x %d", path, h.naxes[0],
                count / (h.naxes[0] ? h.naxes[0] : 1), naxis1, naxis2);
  }
  const int bytes = std::abs(h.bitpix) / 8;
  const bool scaled = h.bscale != 1.0 || h.bzero != 0.0;
  if (fseeko(f, (off_t)h.data_offset, SEEK_SET) != 0) {
    fclose(f);
    return fail("%s: cannot seek to the data", path);
  }
  // 8-byte values are read straight into the image and swapped in place;
  // narrower ones through a staging chunk.
  std::vector<unsigned char> buf(bytes == 8 ? 0 : (size_t)bytes * kChunk);
  for (long long i0 = 0; i0 < count; i0 += (long long)kChunk) {
    const size_t nb = (size_t)std::min((long long)kChunk, count - i0);
    double* out = image + i0;
    unsigned char* src = bytes == 8 ? reinterpret_cast<unsigned char*>(out) : buf.data();
    if (fread(src, (size_t)bytes, nb, f) != nb) {
      fclose(f);
      return fail("%s: the data end early (%lld of %lld values)", path, i0, count);
    }
    // Unit scaling leaves each value as stored, so -0.0 and every other
    // double read back bit for bit.
    decode_chunk(src, nb, h, scaled, out);
  }
  fclose(f);
  return 0;
}

extern "C" int imcom_fits_write(const char* path, int naxis1, int naxis2, const double* image) {
  if (!path) return -1;
  if (naxis1 < 1) return -2;
  if (naxis2 < 1) return -3;
  if (!image) return -4;
  const long long naxes[2] = {naxis1, naxis2};
  return write_image(path, 2, naxes, image);
}

extern "C" int imcom_fits_write_cube(const char* path, int naxis1, int naxis2, int naxis3,
                                     const double* cube) {
  if (!path) return -1;
  if (naxis1 < 1) return -2;
  if (naxis2 < 1) return -3;
  if (naxis3 < 1) return -4;
  if (!cube) return -5;
  const long long naxes[3] = {naxis1, naxis2, naxis3};
  return write_image(path, 3, naxes, cube);
}
