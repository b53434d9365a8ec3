// NIfTI-1 reading and writing (see nifti.h).
#include "nifti.h"

#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

namespace drb {
namespace nifti {
namespace {

// Header field offsets of the NIfTI-1 layout.
enum : int {
  O_SIZEOF_HDR = 0,
  O_DIM = 40,
  O_INTENT_P = 56,
  O_INTENT_CODE = 68,
  O_DATATYPE = 70,
  O_BITPIX = 72,
  O_SLICE_START = 74,
  O_PIXDIM = 76,
  O_VOX_OFFSET = 108,
  O_SCL = 112,
  O_SLICE_END = 120,
  O_CAL = 124,
  O_SLICE_DURATION = 132,
  O_TOFFSET = 136,
  O_GL = 140,
  O_QFORM_CODE = 252,
  O_SFORM_CODE = 254,
  O_QUATERN = 256,
  O_SROW = 280,
  O_MAGIC = 344,
};

template <class T>
T get(const unsigned char* h, int off) {
  T v;
  std::memcpy(&v, h + off, sizeof(T));
  return v;
}
template <class T>
void put(unsigned char* h, int off, T v) {
  std::memcpy(h + off, &v, sizeof(T));
}

void swap_bytes(unsigned char* p, int size, int count) {
  for (int i = 0; i < count; i++, p += size) std::reverse(p, p + size);
}

// Every multi-byte numeric field of the header: (offset, element size, count).
void swap_header(unsigned char* h) {
  static const int fields[][3] = {
      {O_SIZEOF_HDR, 4, 1}, {32, 4, 1},        {36, 2, 1},        {O_DIM, 2, 8},       {O_INTENT_P, 4, 3},
      {O_INTENT_CODE, 2, 1}, {O_DATATYPE, 2, 1}, {O_BITPIX, 2, 1},  {O_SLICE_START, 2, 1}, {O_PIXDIM, 4, 8},
      {O_VOX_OFFSET, 4, 1}, {O_SCL, 4, 2},       {O_SLICE_END, 2, 1}, {O_CAL, 4, 2},       {O_SLICE_DURATION, 4, 1},
      {O_TOFFSET, 4, 1},    {O_GL, 4, 2},        {O_QFORM_CODE, 2, 1}, {O_SFORM_CODE, 2, 1}, {O_QUATERN, 4, 6},
      {O_SROW, 4, 12}};
  for (const auto& f : fields) swap_bytes(h + f[0], f[1], f[2]);
}

bool ends_with(const std::string& s, const std::string& t) {
  return s.size() >= t.size() && s.compare(s.size() - t.size(), t.size(), t) == 0;
}

struct GzFile {
  gzFile f = nullptr;
  explicit GzFile(const std::string& path, const char* mode) { f = gzopen(path.c_str(), mode); }
  ~GzFile() {
    if (f) gzclose(f);
  }
  bool read_exact(void* dst, size_t n) {
    unsigned char* p = (unsigned char*)dst;
    while (n > 0) {
      const unsigned chunk = (unsigned)std::min<size_t>(n, 1u << 30);
      const int got = gzread(f, p, chunk);
      if (got <= 0) return false;
      p += got;
      n -= (size_t)got;
    }
    return true;
  }
  bool write_exact(const void* src, size_t n) {
    const unsigned char* p = (const unsigned char*)src;
    while (n > 0) {
      const unsigned chunk = (unsigned)std::min<size_t>(n, 1u << 30);
      const int put_n = gzwrite(f, p, chunk);
      if (put_n <= 0) return false;
      p += put_n;
      n -= (size_t)put_n;
    }
    return true;
  }
};

bool read_header(const std::string& path, unsigned char* h, bool* swapped) {
  GzFile g(path, "rb");
  if (!g.f || !g.read_exact(h, 348)) return false;
  int32_t sz = get<int32_t>(h, O_SIZEOF_HDR);
  *swapped = false;
  if (sz != 348) {
    swap_bytes((unsigned char*)&sz, 4, 1);
    if (sz != 348) return false;
    swap_header(h);
    *swapped = true;
  }
  const char* m = (const char*)h + O_MAGIC;
  return (std::memcmp(m, "n+1\0", 4) == 0 || std::memcmp(m, "ni1\0", 4) == 0);
}

// Header and data file names of a dataset.
void dataset_files(const std::string& path, std::string* hdr, std::string* img) {
  std::string base = path;
  bool gz = false;
  if (ends_with(base, ".gz")) {
    base = base.substr(0, base.size() - 3);
    gz = true;
  }
  if (ends_with(base, ".img")) {
    const std::string stem = base.substr(0, base.size() - 4);
    *hdr = stem + ".hdr" + (gz ? ".gz" : "");
    *img = path;
  } else if (ends_with(base, ".hdr")) {
    const std::string stem = base.substr(0, base.size() - 4);
    *hdr = path;
    *img = stem + ".img" + (gz ? ".gz" : "");
  } else {
    *hdr = path;
    *img = path;
  }
}

// qto_xyz from the header: quaternion form when qform_code > 0, pixel-size
// diagonal otherwise (the two index-to-space methods of the NIfTI-1 format).
void compute_qform(Image* im) {
  const unsigned char* h = im->hdr;
  double m[4][4] = {{0}};
  m[3][3] = 1.0;
  auto psize = [&](int k) {
    const double d = (double)im->pixdim[k];
    return d > 0 ? d : 1.0;
  };
  if (im->qform_code > 0) {
    double b = get<float>(h, O_QUATERN + 0), c = get<float>(h, O_QUATERN + 4), d = get<float>(h, O_QUATERN + 8);
    const double qx = get<float>(h, O_QUATERN + 12), qy = get<float>(h, O_QUATERN + 16),
                 qz = get<float>(h, O_QUATERN + 20);
    double s = b * b + c * c + d * d, a;
    if (s >= 1.0) {  // a 180-degree rotation: renormalise (b, c, d), a = 0
      const double r = 1.0 / std::sqrt(s);
      b *= r; c *= r; d *= r;
      a = 0.0;
    } else {
      a = std::sqrt(1.0 - s);
    }
    const double R[3][3] = {{a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)},
                            {2 * (b * c + a * d), a * a + c * c - b * b - d * d, 2 * (c * d - a * b)},
                            {2 * (b * d - a * c), 2 * (c * d + a * b), a * a + d * d - b * b - c * c}};
    const double qfac = im->pixdim[0] < 0 ? -1.0 : 1.0;
    const double sc[3] = {psize(1), psize(2), psize(3) * qfac};
    const double off[3] = {qx, qy, qz};
    for (int i = 0; i < 3; i++) {
      for (int j = 0; j < 3; j++) m[i][j] = R[i][j] * sc[j];
      m[i][3] = off[i];
    }
  } else {
    for (int k = 0; k < 3; k++) m[k][k] = psize(k + 1);
  }
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) im->qto_xyz[4 * i + j] = (float)m[i][j];
}

template <class T>
void convert(const unsigned char* src, size_t n, bool swapped, std::vector<float>* out) {
  out->resize(n);
  for (size_t i = 0; i < n; i++) {
    unsigned char b[sizeof(T)];
    std::memcpy(b, src + i * sizeof(T), sizeof(T));
    if (swapped) std::reverse(b, b + sizeof(T));
    T v;
    std::memcpy(&v, b, sizeof(T));
    (*out)[i] = (float)v;
  }
}

}  // namespace

bool is_nifti_file(const std::string& path) {
  std::string hdr, img;
  dataset_files(path, &hdr, &img);
  unsigned char h[348];
  bool sw;
  return read_header(hdr, h, &sw);
}

Image read(const std::string& path) {
  Image im;
  im.fname = path;
  std::string hdr_path, img_path;
  dataset_files(path, &hdr_path, &img_path);
  bool swapped = false;
  if (!read_header(hdr_path, im.hdr, &swapped))
    throw std::runtime_error("not a NIfTI-1 file: " + path);
  for (int k = 0; k < 8; k++) {
    im.dim[k] = get<int16_t>(im.hdr, O_DIM + 2 * k);
    im.pixdim[k] = get<float>(im.hdr, O_PIXDIM + 4 * k);
  }
  if (im.dim[0] < 1 || im.dim[0] > 7) throw std::runtime_error("bad NIfTI dim[0] in " + path);
  for (int k = 1; k <= std::min(im.dim[0], 3); k++)
    if (im.dim[k] < 1) throw std::runtime_error("bad NIfTI dimension in " + path);
  for (int k = im.dim[0] + 1; k <= 3; k++) im.dim[k] = 1;
  im.datatype = get<int16_t>(im.hdr, O_DATATYPE);
  im.qform_code = get<int16_t>(im.hdr, O_QFORM_CODE);
  im.sform_code = get<int16_t>(im.hdr, O_SFORM_CODE);
  compute_qform(&im);

  size_t esize = 0;
  switch (im.datatype) {
    case DT_UINT8: case DT_INT8: esize = 1; break;
    case DT_INT16: case DT_UINT16: esize = 2; break;
    case DT_INT32: case DT_UINT32: case DT_FLOAT32: esize = 4; break;
    case DT_FLOAT64: case DT_INT64: case DT_UINT64: esize = 8; break;
    default: throw std::runtime_error("unsupported NIfTI data type " + std::to_string(im.datatype) + " in " + path);
  }
  const size_t n = (size_t)im.dim[1] * im.dim[2] * im.dim[3];
  const bool single = std::memcmp(im.hdr + O_MAGIC, "n+1\0", 4) == 0;
  const float vo = get<float>(im.hdr, O_VOX_OFFSET);
  size_t offset = single ? (size_t)std::max(vo, 352.0f) : (size_t)std::max(vo, 0.0f);
  std::vector<unsigned char> raw(n * esize);
  {
    GzFile g(single ? hdr_path : img_path, "rb");
    if (!g.f) throw std::runtime_error("cannot open NIfTI data file for " + path);
    if (offset > 0 && gzseek(g.f, (z_off_t)offset, SEEK_SET) < 0) throw std::runtime_error("bad vox_offset in " + path);
    if (!g.read_exact(raw.data(), raw.size())) throw std::runtime_error("truncated NIfTI data in " + path);
  }
  switch (im.datatype) {
    case DT_UINT8: convert<uint8_t>(raw.data(), n, swapped, &im.data); break;
    case DT_INT8: convert<int8_t>(raw.data(), n, swapped, &im.data); break;
    case DT_INT16: convert<int16_t>(raw.data(), n, swapped, &im.data); break;
    case DT_UINT16: convert<uint16_t>(raw.data(), n, swapped, &im.data); break;
    case DT_INT32: convert<int32_t>(raw.data(), n, swapped, &im.data); break;
    case DT_UINT32: convert<uint32_t>(raw.data(), n, swapped, &im.data); break;
    case DT_FLOAT32: convert<float>(raw.data(), n, swapped, &im.data); break;
    case DT_FLOAT64: convert<double>(raw.data(), n, swapped, &im.data); break;
    case DT_INT64: convert<int64_t>(raw.data(), n, swapped, &im.data); break;
    case DT_UINT64: convert<uint64_t>(raw.data(), n, swapped, &im.data); break;
    default: break;
  }
  return im;
}

void write(const Image& geom, const std::vector<float>& values, const std::string& path) {
  if (values.size() != geom.nvox()) throw std::runtime_error("nifti::write: value count differs from the grid");
  unsigned char h[348];
  std::memcpy(h, geom.hdr, 348);
  const bool dbl = geom.datatype == DT_FLOAT64;
  put<int32_t>(h, O_SIZEOF_HDR, 348);
  put<int16_t>(h, O_DATATYPE, dbl ? (int16_t)DT_FLOAT64 : (int16_t)DT_FLOAT32);
  put<int16_t>(h, O_BITPIX, dbl ? (int16_t)64 : (int16_t)32);
  const int nd = std::min(std::max(geom.dim[0], 1), 3);
  put<int16_t>(h, O_DIM, (int16_t)nd);
  for (int k = nd + 1; k < 8; k++) put<int16_t>(h, O_DIM + 2 * k, (int16_t)1);
  put<float>(h, O_VOX_OFFSET, 352.0f);
  std::memcpy(h + O_MAGIC, "n+1\0", 4);
  const bool gz = ends_with(path, ".gz");
  GzFile g(path, gz ? "wb6" : "wbT");
  if (!g.f) throw std::runtime_error("cannot write " + path);
  const unsigned char ext[4] = {0, 0, 0, 0};
  bool ok = g.write_exact(h, 348) && g.write_exact(ext, 4);
  if (dbl) {
    std::vector<double> d(values.begin(), values.end());
    ok = ok && g.write_exact(d.data(), d.size() * sizeof(double));
  } else {
    ok = ok && g.write_exact(values.data(), values.size() * sizeof(float));
  }
  if (!ok) throw std::runtime_error("write failed: " + path);
}

bool same_orientation(const Image& a, const Image& b, float tol) {
  float m = 0.f;
  for (int i = 0; i < 16; i++) m = std::max(m, std::fabs(a.qto_xyz[i] - b.qto_xyz[i]));
  return m <= tol;
}

}  // namespace nifti
}  // namespace drb
