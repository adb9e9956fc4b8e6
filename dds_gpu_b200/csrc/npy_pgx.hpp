// Reader of Pgx DDS result files (.npy, little-endian int32, shape (2, n, 4)): row 0 holds
// the deals, row 1 the DDS tables. The encoding is the dataset's (decoded by the
// reference in src/npy.h:47-63, kept so the same files are read):
//   key[suit]: 2-bit owner of each card, card A,2,3..K at shift 2*(12-i), suits S,H,D,C;
//   value[seat]: 4-bit tricks per strain, strain C,D,H,S,NT at shift 4*(4-strain).
#pragma once
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

namespace pgx {

// Deals [start, start+count): hands (4 per deal) and tables tricks[i*20 + strain*4 + seat].
inline bool load(const char* path, long start, long count, std::vector<uint64_t>& hands,
                 std::vector<uint8_t>& tricks, std::string& err) {
  FILE* f = fopen(path, "rb");
  if (!f) {
    err = "cannot open";
    return false;
  }
  unsigned char pre[12];
  if (fread(pre, 1, 10, f) != 10 || memcmp(pre, "\x93NUMPY", 6) != 0) {
    fclose(f);
    err = "not an .npy file";
    return false;
  }
  long hlen, data;
  if (pre[6] == 1) {
    hlen = pre[8] | (pre[9] << 8);
    data = 10 + hlen;
  } else {
    if (fread(pre + 10, 1, 2, f) != 2) {
      fclose(f);
      err = "short header";
      return false;
    }
    hlen = (long)pre[8] | ((long)pre[9] << 8) | ((long)pre[10] << 16) | ((long)pre[11] << 24);
    data = 12 + hlen;
  }
  std::string hdr(hlen, '\0');
  if (fread(&hdr[0], 1, hlen, f) != (size_t)hlen) {
    fclose(f);
    err = "short header";
    return false;
  }
  size_t sp = hdr.find("'shape': (2, ");
  if (sp == std::string::npos || hdr.find("<i4") == std::string::npos ||
      hdr.find("'fortran_order': False") == std::string::npos) {
    fclose(f);
    err = "expected int32 C-order array of shape (2, n, 4)";
    return false;
  }
  long total = atol(hdr.c_str() + sp + 13);
  if (start < 0) start += total;
  if (start < 0 || count < 0 || start + count > total) {
    fclose(f);
    err = "range outside the file";
    return false;
  }
  std::vector<int32_t> keys((size_t)count * 4), vals((size_t)count * 4);
  bool ok = fseek(f, data + start * 16, SEEK_SET) == 0 &&
            fread(keys.data(), 16, count, f) == (size_t)count &&
            fseek(f, data + (total + start) * 16, SEEK_SET) == 0 &&
            fread(vals.data(), 16, count, f) == (size_t)count;
  fclose(f);
  if (!ok && count > 0) {
    err = "short data";
    return false;
  }
  hands.assign((size_t)count * 4, 0);
  tricks.assign((size_t)count * 20, 0);
  for (long i = 0; i < count; i++) {
    for (int s = 0; s < 4; s++) {
      uint32_t key = (uint32_t)keys[i * 4 + s];
      for (int k = 0; k < 13; k++) {
        int seat = (key >> (2 * (12 - k))) & 3;
        int rank = k == 0 ? 12 : k - 1;  // A first, then 2..K
        hands[i * 4 + seat] |= 1ull << (s * 16 + rank);
      }
    }
    for (int seat = 0; seat < 4; seat++)
      for (int strain = 0; strain < 5; strain++)
        tricks[i * 20 + strain * 4 + seat] = (uint8_t)(((uint32_t)vals[i * 4 + seat] >> (4 * (4 - strain))) & 15);
  }
  return true;
}

}  // namespace pgx
