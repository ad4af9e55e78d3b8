// NIfTI-1 single-file (.nii / .nii.gz) reader and writer, see nifti_io.h.
#include "nifti_io.h"

#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <stdexcept>
#include <system_error>
#include <thread>
#include <vector>

namespace nifti {
namespace {

#pragma pack(push, 1)
struct Header {
  int32_t sizeof_hdr;
  char data_type[10];
  char db_name[18];
  int32_t extents;
  int16_t session_error;
  char regular;
  char dim_info;
  int16_t dim[8];
  float intent_p1, intent_p2, intent_p3;
  int16_t intent_code, datatype, bitpix, slice_start;
  float pixdim[8];
  float vox_offset, scl_slope, scl_inter;
  int16_t slice_end;
  char slice_code, xyzt_units;
  float cal_max, cal_min, slice_duration, toffset;
  int32_t glmax, glmin;
  char descrip[80];
  char aux_file[24];
  int16_t qform_code, sform_code;
  float quatern_b, quatern_c, quatern_d, qoffset_x, qoffset_y, qoffset_z;
  float srow_x[4], srow_y[4], srow_z[4];
  char intent_name[16];
  char magic[4];
};
#pragma pack(pop)
static_assert(sizeof(Header) == 348, "NIfTI-1 header is 348 bytes");

template <class T>
void swap_bytes(T& v) {
  unsigned char* p = reinterpret_cast<unsigned char*>(&v);
  for (size_t i = 0; i < sizeof(T) / 2; ++i) std::swap(p[i], p[sizeof(T) - 1 - i]);
}

void swap_header(Header& h) {
  swap_bytes(h.sizeof_hdr);
  swap_bytes(h.extents);
  swap_bytes(h.session_error);
  for (auto& d : h.dim) swap_bytes(d);
  swap_bytes(h.intent_p1);
  swap_bytes(h.intent_p2);
  swap_bytes(h.intent_p3);
  swap_bytes(h.intent_code);
  swap_bytes(h.datatype);
  swap_bytes(h.bitpix);
  swap_bytes(h.slice_start);
  for (auto& p : h.pixdim) swap_bytes(p);
  swap_bytes(h.vox_offset);
  swap_bytes(h.scl_slope);
  swap_bytes(h.scl_inter);
  swap_bytes(h.slice_end);
  swap_bytes(h.cal_max);
  swap_bytes(h.cal_min);
  swap_bytes(h.slice_duration);
  swap_bytes(h.toffset);
  swap_bytes(h.glmax);
  swap_bytes(h.glmin);
  swap_bytes(h.qform_code);
  swap_bytes(h.sform_code);
  swap_bytes(h.quatern_b);
  swap_bytes(h.quatern_c);
  swap_bytes(h.quatern_d);
  swap_bytes(h.qoffset_x);
  swap_bytes(h.qoffset_y);
  swap_bytes(h.qoffset_z);
  for (int k = 0; k < 4; ++k) {
    swap_bytes(h.srow_x[k]);
    swap_bytes(h.srow_y[k]);
    swap_bytes(h.srow_z[k]);
  }
}

struct GzReader {
  gzFile f;
  explicit GzReader(const std::string& p) : f(gzopen(p.c_str(), "rb")) {
    if (!f) throw std::runtime_error("cannot open " + p);
  }
  ~GzReader() { gzclose(f); }
  void read(void* dst, size_t n, const std::string& what) {
    unsigned char* d = static_cast<unsigned char*>(dst);
    while (n > 0) {
      const unsigned chunk = (unsigned)std::min<size_t>(n, 1u << 30);
      int got = gzread(f, d, chunk);
      if (got <= 0) throw std::runtime_error("short read in " + what);
      d += got;
      n -= (size_t)got;
    }
  }
};

bool ends_with(const std::string& s, const std::string& suf) {
  return s.size() >= suf.size() && s.compare(s.size() - suf.size(), suf.size(), suf) == 0;
}

// bytes as one gzip member (deflate level 6, the level the single-stream writer used)
bool gzip_member(const unsigned char* src, size_t n, std::vector<unsigned char>& out) {
  z_stream z;
  std::memset(&z, 0, sizeof(z));
  if (deflateInit2(&z, 6, Z_DEFLATED, 15 + 16, 8, Z_DEFAULT_STRATEGY) != Z_OK) return false;
  out.resize(deflateBound(&z, (uLong)n) + 64);
  z.next_in = const_cast<unsigned char*>(src);
  z.avail_in = (uInt)n;
  z.next_out = out.data();
  z.avail_out = (uInt)out.size();
  const int rc = deflate(&z, Z_FINISH);
  out.resize(z.total_out);
  deflateEnd(&z);
  return rc == Z_STREAM_END;
}

// A .gz file as consecutive gzip members of 8 MB of input each, compressed over the host's threads and
// written in order.  A multi-member file is one gzip stream to its readers (zlib's gzread, which
// niftilib's znzlib and this reader use, gunzip, Python's gzip); the decompressed bytes are those of a
// single member, and a field of 87 MB compresses in well under a second instead of about five.
void write_gzip_members(const std::string& path, const std::vector<unsigned char>& all) {
  constexpr size_t kChunk = size_t(8) << 20;
  const size_t chunks = std::max<size_t>(1, (all.size() + kChunk - 1) / kChunk);
  const unsigned hw = (unsigned)std::min<size_t>(chunks, std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
  std::FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("cannot write " + path);
  bool ok = true;
  std::vector<std::vector<unsigned char>> out(hw);
  std::vector<char> done(hw, 0);
  for (size_t c0 = 0; ok && c0 < chunks; c0 += hw) {
    const unsigned wave = (unsigned)std::min<size_t>(hw, chunks - c0);
    auto part = [&](unsigned t) {
      const size_t b = (c0 + t) * kChunk, e = std::min(all.size(), b + kChunk);
      try {
        done[t] = gzip_member(all.data() + b, e - b, out[t]) ? 1 : 0;
      } catch (const std::bad_alloc&) {
        done[t] = 0;  // reported as a failed write, not thrown across the thread
      }
    };
    std::vector<std::thread> pool;
    unsigned started = 1;
    try {
      for (; started < wave; ++started) pool.emplace_back(part, started);
    } catch (const std::system_error&) {
      // no more threads: the chunks not started are compressed here
    }
    part(0);
    for (unsigned t = started; t < wave; ++t) part(t);
    for (std::thread& th : pool) th.join();
    for (unsigned t = 0; ok && t < wave; ++t)
      ok = done[t] && std::fwrite(out[t].data(), 1, out[t].size(), f) == out[t].size();
  }
  if (std::fclose(f) != 0 || !ok) throw std::runtime_error("write failed: " + path);
}

}  // namespace

Image read(const std::string& path) {
  GzReader r(path);
  Header h;
  r.read(&h, sizeof(h), path);
  bool swapped = false;
  if (h.sizeof_hdr != 348) {
    swap_header(h);
    swapped = true;
    if (h.sizeof_hdr != 348) throw std::runtime_error(path + ": not a NIfTI-1 file");
  }
  if (std::memcmp(h.magic, "n+1", 3) != 0) throw std::runtime_error(path + ": only single-file NIfTI-1 is supported");
  Image img;
  const int nd = h.dim[0];
  if (nd < 1 || nd > 7) throw std::runtime_error(path + ": bad dim[0]");
  long long n[7] = {1, 1, 1, 1, 1, 1, 1};
  for (int k = 1; k <= nd; ++k) n[k - 1] = h.dim[k] > 0 ? h.dim[k] : 1;
  img.size[0] = n[0];
  img.size[1] = n[1];
  img.size[2] = n[2];
  img.components = (int)(n[4]);
  img.dim = (n[2] > 1) ? 3 : 2;
  if (n[3] != 1) {  // a 4-D series: its volumes are held as component planes
    if (n[4] != 1) throw std::runtime_error(path + ": time series of vector images are not supported");
    img.time_series = true;
    img.components = (int)n[3];
    img.time_step = h.pixdim[4] > 0 ? h.pixdim[4] : 1.0;
  }
  if (n[5] != 1 || n[6] != 1) throw std::runtime_error(path + ": dimensions 6 and 7 are not supported");
  for (int k = 0; k < 3; ++k) img.spacing[k] = h.pixdim[k + 1] > 0 ? h.pixdim[k + 1] : 1.0;
  // RAS affine
  double A[3][4];
  if (h.sform_code > 0) {
    for (int c = 0; c < 4; ++c) {
      A[0][c] = h.srow_x[c];
      A[1][c] = h.srow_y[c];
      A[2][c] = h.srow_z[c];
    }
  } else if (h.qform_code > 0) {
    double b = h.quatern_b, c = h.quatern_c, d = h.quatern_d;
    double a = 1.0 - (b * b + c * c + d * d);
    a = a < 1e-7 ? 0.0 : std::sqrt(a);
    const double qfac = h.pixdim[0] < 0 ? -1.0 : 1.0;
    const double R[3][3] = {{a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)},
                            {2 * (b * c + a * d), a * a + c * c - b * b - d * d, 2 * (c * d - a * b)},
                            {2 * (b * d - a * c), 2 * (c * d + a * b), a * a + d * d - c * c - b * b}};
    for (int rr = 0; rr < 3; ++rr) {
      A[rr][0] = R[rr][0] * img.spacing[0];
      A[rr][1] = R[rr][1] * img.spacing[1];
      A[rr][2] = R[rr][2] * img.spacing[2] * qfac;
    }
    A[0][3] = h.qoffset_x;
    A[1][3] = h.qoffset_y;
    A[2][3] = h.qoffset_z;
  } else {
    for (int rr = 0; rr < 3; ++rr)
      for (int c = 0; c < 4; ++c) A[rr][c] = (rr == c) ? img.spacing[rr] : 0.0;
  }
  // RAS -> LPS, direction columns normalised by spacing
  for (int c = 0; c < 4; ++c) {
    A[0][c] = -A[0][c];
    A[1][c] = -A[1][c];
  }
  for (int k = 0; k < 3; ++k) img.origin[k] = A[k][3];
  for (int c = 0; c < 3; ++c) {
    double nrm = std::sqrt(A[0][c] * A[0][c] + A[1][c] * A[1][c] + A[2][c] * A[2][c]);
    if (nrm <= 0) nrm = 1.0;
    for (int rr = 0; rr < 3; ++rr) img.direction[rr * 3 + c] = A[rr][c] / nrm;
  }
  // payload: the element size comes from the datatype, as niftilib takes it (bitpix is not used), and
  // the data are read in bounded chunks, so a header that claims more data than the file holds fails
  // on the short read instead of allocating what it claims
  int bytes = 0;
  switch (h.datatype) {
    case 2: case 256: bytes = 1; break;
    case 4: case 512: bytes = 2; break;
    case 8: case 16: case 768: bytes = 4; break;
    case 64: bytes = 8; break;
    default: throw std::runtime_error(path + ": unsupported NIfTI datatype " + std::to_string(h.datatype));
  }
  const long long count = img.voxels() * img.components;
  if (!(h.vox_offset < (float)(1 << 26))) throw std::runtime_error(path + ": vox_offset out of range");
  const size_t off = (size_t)(h.vox_offset > 352 ? h.vox_offset : 352);
  std::vector<unsigned char> skip(off - sizeof(h));
  if (!skip.empty()) r.read(skip.data(), skip.size(), path);
  const size_t total = (size_t)count * (size_t)bytes, chunk = (size_t)1 << 26;
  std::vector<unsigned char> raw;
  for (size_t done = 0; done < total; done += std::min(chunk, total - done)) {
    raw.resize(done + std::min(chunk, total - done));
    r.read(raw.data() + done, raw.size() - done, path);
  }
  img.data.resize((size_t)count);
  auto conv = [&](auto tag) {
    using T = decltype(tag);
    for (long long i = 0; i < count; ++i) {
      T v;
      std::memcpy(&v, raw.data() + (size_t)i * sizeof(T), sizeof(T));
      if (swapped) swap_bytes(v);
      img.data[(size_t)i] = (float)v;
    }
  };
  switch (h.datatype) {
    case 2: conv(uint8_t()); break;
    case 4: conv(int16_t()); break;
    case 8: conv(int32_t()); break;
    case 16: conv(float()); break;
    case 64: conv(double()); break;
    case 256: conv(int8_t()); break;
    case 512: conv(uint16_t()); break;
    case 768: conv(uint32_t()); break;
    default: throw std::runtime_error(path + ": unsupported NIfTI datatype " + std::to_string(h.datatype));
  }
  if (h.scl_slope != 0.0f && !(h.scl_slope == 1.0f && h.scl_inter == 0.0f))
    for (auto& v : img.data) v = v * h.scl_slope + h.scl_inter;
  return img;
}

void write(const std::string& path, const Image& img) {
  Header h;
  std::memset(&h, 0, sizeof(h));
  h.sizeof_hdr = 348;
  h.regular = 'r';
  const bool series = img.time_series;
  const bool vec = img.components > 1 && !series;
  h.dim[0] = series ? 4 : vec ? 5 : (img.dim == 3 ? 3 : 2);
  h.dim[1] = (int16_t)img.size[0];
  h.dim[2] = (int16_t)img.size[1];
  h.dim[3] = (int16_t)(img.dim == 3 ? img.size[2] : 1);
  h.dim[4] = (int16_t)(series ? img.components : 1);
  h.dim[5] = (int16_t)(series ? 1 : img.components);
  h.dim[6] = h.dim[7] = 1;
  if (vec) h.intent_code = 1007;  // NIFTI_INTENT_VECTOR
  int out_bytes = 0;
  switch (img.out_datatype) {
    case 2: case 256: out_bytes = 1; break;
    case 4: out_bytes = 2; break;
    case 8: case 16: out_bytes = 4; break;
    case 64: out_bytes = 8; break;
    default: throw std::runtime_error(path + ": unsupported output datatype " + std::to_string(img.out_datatype));
  }
  h.datatype = (int16_t)img.out_datatype;
  h.bitpix = (int16_t)(8 * out_bytes);
  h.pixdim[0] = 1.0f;
  for (int k = 0; k < 3; ++k) h.pixdim[k + 1] = (float)(k < img.dim ? img.spacing[k] : 1.0);
  h.pixdim[4] = (float)(series ? img.time_step : 1.0);
  h.pixdim[5] = h.pixdim[6] = h.pixdim[7] = 1.0f;
  h.vox_offset = 352.0f;
  h.scl_slope = 1.0f;
  h.xyzt_units = 2 | 8;  // mm, s
  std::strncpy(h.descrip, "synx", sizeof(h.descrip) - 1);
  std::memcpy(h.magic, "n+1\0", 4);
  // LPS geometry -> RAS affine
  double D[3][3];
  for (int rr = 0; rr < 3; ++rr)
    for (int c = 0; c < 3; ++c) D[rr][c] = img.direction[rr * 3 + c];
  if (img.dim == 2) {
    D[0][2] = D[1][2] = D[2][0] = D[2][1] = 0.0;
    D[2][2] = 1.0;
  }
  double A[3][4];
  for (int rr = 0; rr < 3; ++rr) {
    const double sgn = rr < 2 ? -1.0 : 1.0;
    for (int c = 0; c < 3; ++c) A[rr][c] = sgn * D[rr][c] * (c < img.dim ? img.spacing[c] : 1.0);
    A[rr][3] = sgn * (rr < img.dim ? img.origin[rr] : 0.0);
  }
  h.sform_code = 1;
  h.qform_code = 1;
  for (int c = 0; c < 4; ++c) {
    h.srow_x[c] = (float)A[0][c];
    h.srow_y[c] = (float)A[1][c];
    h.srow_z[c] = (float)A[2][c];
  }
  // quaternion of the RAS rotation (columns normalised); a left-handed frame sets qfac = -1
  double R[3][3];
  for (int rr = 0; rr < 3; ++rr)
    for (int c = 0; c < 3; ++c) R[rr][c] = (rr < 2 ? -1.0 : 1.0) * D[rr][c];
  const double det = R[0][0] * (R[1][1] * R[2][2] - R[1][2] * R[2][1]) -
                     R[0][1] * (R[1][0] * R[2][2] - R[1][2] * R[2][0]) +
                     R[0][2] * (R[1][0] * R[2][1] - R[1][1] * R[2][0]);
  if (det < 0) {
    h.pixdim[0] = -1.0f;
    for (int rr = 0; rr < 3; ++rr) R[rr][2] = -R[rr][2];
  }
  double a = 1.0 + R[0][0] + R[1][1] + R[2][2], b, c, d;
  if (a > 0.5) {
    a = 0.5 * std::sqrt(a);
    b = 0.25 * (R[2][1] - R[1][2]) / a;
    c = 0.25 * (R[0][2] - R[2][0]) / a;
    d = 0.25 * (R[1][0] - R[0][1]) / a;
  } else {
    const double xd = 1.0 + R[0][0] - (R[1][1] + R[2][2]), yd = 1.0 + R[1][1] - (R[0][0] + R[2][2]),
                 zd = 1.0 + R[2][2] - (R[0][0] + R[1][1]);
    if (xd > 1.0) {
      b = 0.5 * std::sqrt(xd);
      c = 0.25 * (R[0][1] + R[1][0]) / b;
      d = 0.25 * (R[0][2] + R[2][0]) / b;
      a = 0.25 * (R[2][1] - R[1][2]) / b;
    } else if (yd > 1.0) {
      c = 0.5 * std::sqrt(yd);
      b = 0.25 * (R[0][1] + R[1][0]) / c;
      d = 0.25 * (R[1][2] + R[2][1]) / c;
      a = 0.25 * (R[0][2] - R[2][0]) / c;
    } else {
      d = 0.5 * std::sqrt(zd);
      b = 0.25 * (R[0][2] + R[2][0]) / d;
      c = 0.25 * (R[1][2] + R[2][1]) / d;
      a = 0.25 * (R[1][0] - R[0][1]) / d;
    }
    if (a < 0.0) {
      b = -b;
      c = -c;
      d = -d;
    }
  }
  h.quatern_b = (float)b;
  h.quatern_c = (float)c;
  h.quatern_d = (float)d;
  h.qoffset_x = (float)A[0][3];
  h.qoffset_y = (float)A[1][3];
  h.qoffset_z = (float)A[2][3];

  const bool gz = ends_with(path, ".gz");
  const char ext[4] = {0, 0, 0, 0};
  // the payload in the output type: floats as they are, doubles widened, integers as a C++ cast of the
  // value truncated toward zero (the reference's CastImageFilter), NaN as 0
  std::vector<unsigned char> conv;
  const unsigned char* p = reinterpret_cast<const unsigned char*>(img.data.data());
  if (img.out_datatype != 16) {
    conv.resize(img.data.size() * (size_t)out_bytes);
    for (size_t i = 0; i < img.data.size(); ++i) {
      const float v = img.data[i];
      unsigned char* q = conv.data() + i * (size_t)out_bytes;
      if (img.out_datatype == 64) {
        const double d = v;
        std::memcpy(q, &d, 8);
        continue;
      }
      const long long t = std::isfinite(v) && std::fabs(v) < 9.0e18f ? (long long)std::trunc(v) : 0;
      switch (img.out_datatype) {
        case 2: { const uint8_t x = (uint8_t)t; std::memcpy(q, &x, 1); break; }
        case 256: { const int8_t x = (int8_t)t; std::memcpy(q, &x, 1); break; }
        case 4: { const int16_t x = (int16_t)t; std::memcpy(q, &x, 2); break; }
        default: { const int32_t x = (int32_t)t; std::memcpy(q, &x, 4); break; }
      }
    }
    p = conv.data();
  }
  const size_t payload = img.data.size() * (size_t)out_bytes;
  if (gz) {
    // header, extension flag and payload as one byte stream, compressed in parallel
    std::vector<unsigned char> all;
    all.reserve(sizeof(h) + 4 + payload);
    const unsigned char* hb = reinterpret_cast<const unsigned char*>(&h);
    all.insert(all.end(), hb, hb + sizeof(h));
    all.insert(all.end(), ext, ext + 4);
    all.insert(all.end(), p, p + payload);
    write_gzip_members(path, all);
    return;
  }
  std::FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("cannot write " + path);
  bool ok = std::fwrite(&h, 1, sizeof(h), f) == sizeof(h) && std::fwrite(ext, 1, 4, f) == 4;
  if (ok && payload) ok = std::fwrite(p, 1, payload, f) == payload;
  if (std::fclose(f) != 0 || !ok) throw std::runtime_error("write failed: " + path);
}

}  // namespace nifti
