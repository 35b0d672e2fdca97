// me_fits.cpp -- the FITS primary-HDU I/O of the inversion driver.
//
// The reference reads and writes through cfitsio (Src/IO.c:120-742); the
// calls it makes are a small subset: the primary array's dimensions and
// BITPIX, reads of doubles from a pixel offset (with BSCALE / BZERO applied,
// as cfitsio does for TDOUBLE reads), creation of a BITPIX -64 image, and
// writes of doubles at a pixel offset.  This file implements exactly those
// on the FITS standard (NASA/IAU FITS 4.0: 2880-byte blocks of 80-character
// header cards, big-endian data); no extensions, no compression.
#include <errno.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/me_b200.h"

namespace me {
int record_error(int code, const char *msg);
}

namespace {

constexpr long kBlock = 2880;
constexpr int kCard = 80;

int fail(int code, const std::string &m) { return me::record_error(code, m.c_str()); }

struct Header {
  int bitpix = 0;
  int naxis = 0;
  long naxes[8] = {0};
  double bscale = 1.0, bzero = 0.0;
  long data_offset = 0;  // bytes from the start of the file
  long nelem() const {
    if (naxis == 0) return 0;
    long n = 1;
    for (int i = 0; i < naxis; i++) n *= naxes[i];
    return n;
  }
};

// value field of a card (columns 11-80), without a trailing comment
std::string card_value(const char *card) {
  std::string v(card + 10, kCard - 10);
  bool quoted = false;
  for (size_t i = 0; i < v.size(); i++) {
    if (v[i] == '\'') quoted = !quoted;
    if (v[i] == '/' && !quoted) {
      v.resize(i);
      break;
    }
  }
  size_t a = v.find_first_not_of(' '), b = v.find_last_not_of(' ');
  return a == std::string::npos ? std::string() : v.substr(a, b - a + 1);
}

std::string card_key(const char *card) {
  std::string k(card, 8);
  size_t b = k.find_last_not_of(' ');
  return b == std::string::npos ? std::string() : k.substr(0, b + 1);
}

int read_header(FILE *f, const char *path, Header &h) {
  char block[kBlock];
  bool end = false, simple = false;
  long nblocks = 0;
  int seen_naxis = 0;
  while (!end) {
    if (fread(block, 1, kBlock, f) != (size_t)kBlock)
      return fail(ME_ERR_FORMAT, std::string("truncated FITS header: ") + path);
    for (int c = 0; c < kBlock / kCard; c++) {
      const char *card = block + c * kCard;
      const std::string key = card_key(card);
      if (nblocks == 0 && c == 0) {
        if (key != "SIMPLE" || card_value(card) != "T")
          return fail(ME_ERR_FORMAT, std::string("not a FITS file: ") + path);
        simple = true;
        continue;
      }
      if (key == "END") {
        end = true;
        break;
      }
      if (card[8] != '=' || card[9] != ' ') continue;  // commentary card
      const std::string v = card_value(card);
      if (key == "BITPIX") {
        h.bitpix = atoi(v.c_str());
      } else if (key == "NAXIS") {
        h.naxis = atoi(v.c_str());
        if (h.naxis < 0 || h.naxis > 8)
          return fail(ME_ERR_FORMAT, std::string("bad NAXIS in ") + path);
      } else if (key.compare(0, 5, "NAXIS") == 0 && key.size() > 5) {
        const int i = atoi(key.c_str() + 5);
        if (i >= 1 && i <= 8) {
          h.naxes[i - 1] = atol(v.c_str());
          seen_naxis++;
        }
      } else if (key == "BSCALE") {
        h.bscale = atof(v.c_str());
      } else if (key == "BZERO") {
        h.bzero = atof(v.c_str());
      }
    }
    nblocks++;
  }
  if (!simple) return fail(ME_ERR_FORMAT, std::string("not a FITS file: ") + path);
  if (h.bitpix != 8 && h.bitpix != 16 && h.bitpix != 32 && h.bitpix != 64 && h.bitpix != -32 &&
      h.bitpix != -64)
    return fail(ME_ERR_FORMAT, std::string("bad BITPIX in ") + path);
  for (int i = 0; i < h.naxis; i++)
    if (h.naxes[i] < 0) return fail(ME_ERR_FORMAT, std::string("bad NAXISn in ") + path);
  (void)seen_naxis;
  h.data_offset = nblocks * kBlock;
  return ME_OK;
}

int open_header(const char *path, const char *mode, FILE **fp, Header &h) {
  FILE *f = fopen(path, mode);
  if (!f) return fail(ME_ERR_IO, std::string("cannot open ") + path + ": " + strerror(errno));
  const int rc = read_header(f, path, h);
  if (rc) {
    fclose(f);
    return rc;
  }
  *fp = f;
  return ME_OK;
}

inline uint16_t bswap16(uint16_t v) { return (uint16_t)((v << 8) | (v >> 8)); }
inline uint32_t bswap32(uint32_t v) { return __builtin_bswap32(v); }
inline uint64_t bswap64(uint64_t v) { return __builtin_bswap64(v); }

// n values of the primary array from element `first` on, as doubles
int read_elems(FILE *f, const char *path, const Header &h, long first, long n, double *out) {
  const int bytes = (h.bitpix < 0 ? -h.bitpix : h.bitpix) / 8;
  if (first < 0 || n < 0 || first + n > h.nelem())
    return fail(ME_ERR_ARG, std::string("read outside the image of ") + path);
  if (fseek(f, h.data_offset + first * bytes, SEEK_SET) != 0)
    return fail(ME_ERR_IO, std::string("seek failed in ") + path);
  std::vector<unsigned char> buf;
  const long chunk = 1 << 20;
  for (long done = 0; done < n; done += chunk) {
    const long m = n - done < chunk ? n - done : chunk;
    buf.resize((size_t)m * bytes);
    if (fread(buf.data(), (size_t)bytes, (size_t)m, f) != (size_t)m)
      return fail(ME_ERR_IO, std::string("truncated FITS data: ") + path);
    double *o = out + done;
    const unsigned char *b = buf.data();
    for (long i = 0; i < m; i++, b += bytes) {
      double v;
      switch (h.bitpix) {
        case 8: v = (double)b[0]; break;
        case 16: { uint16_t t; memcpy(&t, b, 2); v = (double)(int16_t)bswap16(t); } break;
        case 32: { uint32_t t; memcpy(&t, b, 4); v = (double)(int32_t)bswap32(t); } break;
        case 64: { uint64_t t; memcpy(&t, b, 8); v = (double)(int64_t)bswap64(t); } break;
        case -32: { uint32_t t; memcpy(&t, b, 4); t = bswap32(t); float x; memcpy(&x, &t, 4); v = x; } break;
        default: { uint64_t t; memcpy(&t, b, 8); t = bswap64(t); memcpy(&v, &t, 8); } break;
      }
      o[i] = h.bzero + h.bscale * v;
    }
  }
  return ME_OK;
}

void put_card(std::string &hdr, const char *key, const std::string &value) {
  char card[kCard + 1];
  snprintf(card, sizeof card, "%-8.8s= %20s", key, value.c_str());
  std::string c(card);
  c.resize(kCard, ' ');
  hdr += c;
}

}  // namespace

extern "C" int me_fits_image_info(const char *path, int *bitpix, int *naxis, long naxes[8]) {
  if (!path) return fail(ME_ERR_ARG, "null path");
  FILE *f = nullptr;
  Header h;
  int rc = open_header(path, "rb", &f, h);
  if (rc) return rc;
  fclose(f);
  if (bitpix) *bitpix = h.bitpix;
  if (naxis) *naxis = h.naxis;
  if (naxes)
    for (int i = 0; i < 8; i++) naxes[i] = i < h.naxis ? h.naxes[i] : 0;
  return ME_OK;
}

extern "C" int me_fits_read(const char *path, long first, long n, double *out) {
  if (!path || (n > 0 && !out)) return fail(ME_ERR_ARG, "null argument");
  FILE *f = nullptr;
  Header h;
  int rc = open_header(path, "rb", &f, h);
  if (rc) return rc;
  rc = read_elems(f, path, h, first, n, out);
  fclose(f);
  return rc;
}

extern "C" int me_fits_create(const char *path, int naxis, const long *naxes) {
  if (!path || !naxes || naxis < 1 || naxis > 8) return fail(ME_ERR_ARG, "bad image shape");
  long n = 1;
  for (int i = 0; i < naxis; i++) {
    if (naxes[i] < 1) return fail(ME_ERR_ARG, "bad image shape");
    n *= naxes[i];
  }
  std::string hdr;
  put_card(hdr, "SIMPLE", "T");
  put_card(hdr, "BITPIX", "-64");
  put_card(hdr, "NAXIS", std::to_string(naxis));
  for (int i = 0; i < naxis; i++) {
    char key[9];
    snprintf(key, sizeof key, "NAXIS%d", i + 1);
    put_card(hdr, key, std::to_string(naxes[i]));
  }
  put_card(hdr, "EXTEND", "T");
  std::string end("END");
  end.resize(kCard, ' ');
  hdr += end;
  hdr.resize((size_t)((hdr.size() + kBlock - 1) / kBlock * kBlock), ' ');
  FILE *f = fopen(path, "wb");
  if (!f) return fail(ME_ERR_IO, std::string("cannot create ") + path + ": " + strerror(errno));
  bool ok = fwrite(hdr.data(), 1, hdr.size(), f) == hdr.size();
  const long data = n * 8, padded = (data + kBlock - 1) / kBlock * kBlock;
  std::vector<char> zeros(1 << 20, 0);
  for (long done = 0; ok && done < padded; done += (long)zeros.size()) {
    const long m = padded - done < (long)zeros.size() ? padded - done : (long)zeros.size();
    ok = fwrite(zeros.data(), 1, (size_t)m, f) == (size_t)m;
  }
  ok = (fclose(f) == 0) && ok;
  if (!ok) return fail(ME_ERR_IO, std::string("short write to ") + path);
  return ME_OK;
}

extern "C" int me_fits_write(const char *path, long first, long n, const double *v) {
  if (!path || (n > 0 && !v)) return fail(ME_ERR_ARG, "null argument");
  FILE *f = nullptr;
  Header h;
  int rc = open_header(path, "r+b", &f, h);
  if (rc) return rc;
  if (h.bitpix != -64) {
    fclose(f);
    return fail(ME_ERR_FORMAT, std::string("writes need a BITPIX -64 image: ") + path);
  }
  if (first < 0 || n < 0 || first + n > h.nelem()) {
    fclose(f);
    return fail(ME_ERR_ARG, std::string("write outside the image of ") + path);
  }
  bool ok = fseek(f, h.data_offset + first * 8, SEEK_SET) == 0;
  std::vector<uint64_t> buf;
  const long chunk = 1 << 20;
  for (long done = 0; ok && done < n; done += chunk) {
    const long m = n - done < chunk ? n - done : chunk;
    buf.resize((size_t)m);
    for (long i = 0; i < m; i++) {
      uint64_t t;
      memcpy(&t, v + done + i, 8);
      buf[i] = bswap64(t);
    }
    ok = fwrite(buf.data(), 8, (size_t)m, f) == (size_t)m;
  }
  ok = (fclose(f) == 0) && ok;
  if (!ok) return fail(ME_ERR_IO, std::string("write failed: ") + path);
  return ME_OK;
}
