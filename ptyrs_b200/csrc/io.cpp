// Scan and reconstruction files (reference ptyrs/src/io/cxi.rs:130-200 `read_cxi`,
// ptyrs/src/io/ptyr.rs `read_ptyr`) on the HDF5 reader of h5.h: the CXI layout PyNX's
// `save_ptycho_data_cxi` writes (counts, translations, energy, distance, pixel sizes, detector
// mask) into a scan the handles take, and the object and probe storages of a PtyPy `.ptyr`.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>

#include "../../include/ptyb200.h"
#include "h5.h"

namespace {

using ptyb::h5::Dataset;
using ptyb::h5::File;
using ptyb::h5::Type;

thread_local std::string g_io_error;

constexpr uint16_t kMasked = 65535, kMaxCount = 65534;
// PyNX's conversion between photon energy and wavelength (reference base/geometry.rs:7-9,
// 134-136): λ = 12.3984 keV·Å / (E / 1.60218e-16 J per keV).
constexpr double kKevAngstrom = 12.3984, kJoulePerKev = 1.60218e-16;

const char* kEnergy = "entry_1/instrument_1/source_1/energy";
const char* kDistance = "entry_1/instrument_1/detector_1/distance";
const char* kXPixel = "entry_1/instrument_1/detector_1/x_pixel_size";
const char* kYPixel = "entry_1/instrument_1/detector_1/y_pixel_size";
const char* kData = "entry_1/data_1/data";
const char* kTranslation = "entry_1/sample_1/geometry_1/translation";
const char* kMask = "entry_1/instrument_1/detector_1/mask";

uint64_t le(const uint8_t* p, int n, bool big) {
  uint64_t v = 0;
  if (big)
    for (int i = 0; i < n; ++i) v = (v << 8) | p[i];
  else
    for (int i = n - 1; i >= 0; --i) v = (v << 8) | p[i];
  return v;
}

// Element i of a dataset of scalars as double (integers of 1, 2, 4 or 8 bytes, floats of 4 or 8,
// enumerations over such integers); any other element size is refused.
double scalar_at(const Type& t, const uint8_t* p) {
  if (t.cls == Type::kEnum) {
    if (!t.base || t.base->cls != Type::kFixed || t.base->size > t.size)
      throw std::runtime_error("an enumeration of an unsupported base type");
    return scalar_at(*t.base, p);
  }
  const bool sized = t.size == 1 || t.size == 2 || t.size == 4 || t.size == 8;
  if (!sized || (t.cls == Type::kFloat && t.size < 4))
    throw std::runtime_error("a dataset of an unsupported element size " +
                             std::to_string(t.size));
  if (t.cls == Type::kFixed) {
    const uint64_t u = le(p, (int)t.size, t.big_endian);
    if (!t.is_signed) return (double)u;
    const int bits = 8 * (int)t.size;
    const int64_t s = bits == 64 ? (int64_t)u : (int64_t)(u << (64 - bits)) >> (64 - bits);
    return (double)s;
  }
  if (t.cls == Type::kFloat) {
    const uint64_t u = le(p, (int)t.size, t.big_endian);
    if (t.size == 4) {
      uint32_t w = (uint32_t)u;
      float f;
      std::memcpy(&f, &w, 4);
      return f;
    }
    if (t.size == 8) {
      double d;
      std::memcpy(&d, &u, 8);
      return d;
    }
  }
  throw std::runtime_error("a dataset of an unsupported element type");
}

std::vector<double> as_f64(const Dataset& d) {
  std::vector<double> out(d.count());
  for (size_t i = 0; i < out.size(); ++i) out[i] = scalar_at(d.type, d.bytes.data() + i * d.type.size);
  return out;
}

double read_scalar(const File& f, const char* path) {
  const Dataset d = f.dataset(path);
  if (d.count() != 1) throw std::runtime_error(std::string(path) + " is not a scalar");
  return as_f64(d)[0];
}

// A complex dataset (a compound of two floats, h5py's complex64 / complex128) as interleaved
// doubles.
std::vector<double> as_c128(const Dataset& d, const std::string& path) {
  const Type& t = d.type;
  if (t.cls != Type::kCompound || t.members.size() != 2 ||
      t.members[0].type->cls != Type::kFloat || t.members[1].type->cls != Type::kFloat)
    throw std::runtime_error(path + " is not complex64 or complex128");
  for (const auto& m : t.members)
    if ((uint64_t)m.offset + m.type->size > t.size)
      throw std::runtime_error(path + ": a member lies outside its element");
  std::vector<double> out(2 * d.count());
  for (size_t i = 0; i < d.count(); ++i)
    for (int k = 0; k < 2; ++k)
      out[2 * i + k] =
          scalar_at(*t.members[k].type, d.bytes.data() + i * t.size + t.members[k].offset);
  return out;
}

template <typename F>
int guarded_io(F&& body) {
  g_io_error.clear();
  try {
    return body();
  } catch (const std::bad_alloc&) {
    g_io_error = "host memory";
    return PTYB_INVALID;
  } catch (const std::exception& e) {
    g_io_error = e.what();
    return PTYB_INVALID;
  }
}

}  // namespace

extern "C" {

int ptyb_read_cxi(const char* path, ptyb_cxi_scan* out) {
  if (!path || !out) return PTYB_INVALID;
  std::memset(out, 0, sizeof(*out));
  return guarded_io([&]() -> int {
    const File f(path);
    const double energy = read_scalar(f, kEnergy), distance = read_scalar(f, kDistance);
    const double px = read_scalar(f, kXPixel), py = read_scalar(f, kYPixel);
    if (px != py)
      throw std::runtime_error("x_pixel_size != y_pixel_size; PyNX assumes square pixels");
    const Dataset data = f.dataset(kData);
    if (data.shape.size() != 3)
      throw std::runtime_error(std::string(kData) + " is not [nframe, ny, nx]");
    const size_t nframe = data.shape[0], ny = data.shape[1], nx = data.shape[2];
    const size_t plane = ny * nx;
    const Dataset tr = f.dataset(kTranslation);
    if (tr.shape.size() != 2 || tr.shape[0] < 2 || tr.shape[1] != nframe)
      throw std::runtime_error(std::string(kTranslation) + " is not [3, nframe]");
    const std::vector<double> t = as_f64(tr);
    std::vector<uint8_t> mask;
    if (f.exists(kMask)) {
      const Dataset m = f.dataset(kMask);
      if (m.shape.size() != 2 || m.shape[0] != ny || m.shape[1] != nx)
        throw std::runtime_error(std::string(kMask) + " is not [ny, nx]");
      for (double v : as_f64(m)) mask.push_back(v != 0.0);
    }
    auto* counts = static_cast<uint16_t*>(std::malloc(nframe * plane * sizeof(uint16_t)));
    auto* y = static_cast<double*>(std::malloc(nframe * sizeof(double)));
    auto* x = static_cast<double*>(std::malloc(nframe * sizeof(double)));
    if (!counts || !y || !x) {
      std::free(counts);
      std::free(y);
      std::free(x);
      throw std::bad_alloc();
    }
    try {
      const bool u16 = data.type.cls == Type::kFixed && data.type.size == 2 && !data.type.is_signed;
      const std::vector<double> vals = u16 ? std::vector<double>() : as_f64(data);
      for (size_t i = 0; i < nframe * plane; ++i) {
        const bool masked = !mask.empty() && mask[i % plane];
        if (u16) {
          // raw counts (reference cxi.rs:178-189): the detector mask marks pixels MASKED
          const uint16_t v = (uint16_t)le(data.bytes.data() + 2 * i, 2, data.type.big_endian);
          counts[i] = masked ? kMasked : v;
          continue;
        }
        // reference base/counts.rs:49-80 (`Counts::from_f64`)
        const double v = vals[i];
        if (masked || v < 0.0) {
          counts[i] = kMasked;
        } else if (!std::isfinite(v) || v > kMaxCount) {
          throw std::runtime_error("count " + std::to_string(v) + " at " + std::to_string(i) +
                                   " is out of range");
        } else if (v != std::floor(v)) {
          throw std::runtime_error("count " + std::to_string(v) + " at " + std::to_string(i) +
                                   " is not an integer");
        } else {
          counts[i] = (uint16_t)v;
        }
      }
    } catch (...) {
      std::free(counts);
      std::free(y);
      std::free(x);
      throw;
    }
    // translation rows: x, y (reference cxi.rs:160-168)
    for (size_t i = 0; i < nframe; ++i) {
      x[i] = t[i];
      y[i] = t[nframe + i];
    }
    out->nframe = (int32_t)nframe;
    out->ny = (int32_t)ny;
    out->nx = (int32_t)nx;
    out->counts = counts;
    out->y = y;
    out->x = x;
    out->wavelength = kKevAngstrom * 1e-10 / (energy / kJoulePerKev);
    out->distance = distance;
    out->detector_pixel = px;
    return PTYB_OK;
  });
}

void ptyb_free_cxi(ptyb_cxi_scan* s) {
  if (!s) return;
  std::free(s->counts);
  std::free(s->y);
  std::free(s->x);
  std::memset(s, 0, sizeof(*s));
}

int ptyb_read_ptyr(const char* path, ptyb_ptyr* out) {
  if (!path || !out) return PTYB_INVALID;
  std::memset(out, 0, sizeof(*out));
  return guarded_io([&]() -> int {
    const File f(path);
    // the one storage under content/<name> (reference ptyr.rs `only_storage`)
    auto storage = [&](const char* name) {
      const std::string c = std::string("content/") + name;
      const auto ids = f.members(c);
      if (ids.size() != 1)
        throw std::runtime_error(c + " holds " + std::to_string(ids.size()) +
                                 " storages, expected one");
      return c + "/" + ids[0];
    };
    const std::string obj = storage("obj"), probe = storage("probe");
    const Dataset od = f.dataset(obj + "/data"), pd = f.dataset(probe + "/data");
    if (od.shape.size() != 3 || pd.shape.size() != 3)
      throw std::runtime_error("storage data is not 3-dimensional");
    const std::vector<double> o = as_c128(od, obj + "/data"), p = as_c128(pd, probe + "/data");
    const std::vector<double> ps = as_f64(f.dataset(obj + "/_psize"));
    const std::vector<double> org = as_f64(f.dataset(obj + "/_origin"));
    if (ps.size() != 2 || org.size() != 2)
      throw std::runtime_error("_psize and _origin must hold [y, x]");
    auto* ob = static_cast<double*>(std::malloc(o.size() * sizeof(double)));
    auto* pb = static_cast<double*>(std::malloc(p.size() * sizeof(double)));
    if (!ob || !pb) {
      std::free(ob);
      std::free(pb);
      throw std::bad_alloc();
    }
    std::memcpy(ob, o.data(), o.size() * sizeof(double));
    std::memcpy(pb, p.data(), p.size() * sizeof(double));
    for (int k = 0; k < 3; ++k) {
      out->obj_shape[k] = (int32_t)od.shape[k];
      out->probe_shape[k] = (int32_t)pd.shape[k];
    }
    out->object = ob;
    out->probe = pb;
    for (int k = 0; k < 2; ++k) {
      out->psize[k] = ps[k];
      out->origin[k] = org[k];
    }
    return PTYB_OK;
  });
}

void ptyb_free_ptyr(ptyb_ptyr* r) {
  if (!r) return;
  std::free(r->object);
  std::free(r->probe);
  std::memset(r, 0, sizeof(*r));
}

const char* ptyb_io_last_error(void) { return g_io_error.c_str(); }

}  // extern "C"
