// gdem_rawdata.cpp -- the RawData post-processing writer and the
// _VelocityMaxMean.dat line of Grains3D over the device state
// (GRAINS_V1/Grains/PostProcessing/src/RawDataPostProcessingWriter.cpp,
// Base/src/Grains.cpp:137-145, 401-408).  Host code on the public C ABI: the
// state, the coordination numbers (counted on the device from the last force
// evaluation) and the velocity reduction come through gdem_download_state,
// gdem_download_coordination and gdem_velocity_stats; this file only formats.
//
// Number format: GrainsExec::doubleToString(ios::scientific, 6, x)
// (Base/src/GrainsExec.cpp:212-224) prints a nonzero x as "%.6e" and a zero
// in the stream's default format ("0", "-0").
#include <cstdio>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "grains_b200.h"

namespace gdem {
void setLastError(std::string const& msg);   // gdem_host.cu: gdem_last_error's text
}  // namespace gdem

namespace {

// the per-time files in the reference's order (prepareResultFiles, :276-318)
const char* const kSuffix[10] = {
    "_position_x.dat", "_position_y.dat", "_position_z.dat",
    "_translational_velocity_x.dat", "_translational_velocity_y.dat",
    "_translational_velocity_z.dat", "_angular_velocity_x.dat",
    "_angular_velocity_y.dat", "_angular_velocity_z.dat", "_coordinationNumber.dat"};

struct RawWriter {
  std::string root;
  bool binary = false;
  FILE* f[10] = {};
  ~RawWriter() {
    for (FILE*& p : f)
      if (p) { std::fclose(p); p = nullptr; }
  }
};

std::mutex g_mu;
std::map<gdem_handle, RawWriter*> g_writers;

void number(std::string& out, double x) {
  char buf[40];
  std::snprintf(buf, sizeof buf, x != 0. ? "%.6e" : "%g", x);
  out += buf;
}

void check(int rc) {
  if (rc != GDEM_OK) throw std::runtime_error(gdem_last_error());
}

void put(FILE* f, const void* p, size_t bytes, std::string const& name) {
  if (bytes && std::fwrite(p, 1, bytes, f) != bytes) throw std::runtime_error("cannot write " + name);
}

// One output time (one_output_Standard, :374-600): every particle, in ID
// order, one column per particle.  All particles of a system are active
// and physical, so the reference's inactive-particle columns (position
// -1e10, zero velocities, class -1) do not occur.
void writeTime(gdem_handle h, RawWriter& w, double time) {
  const int64_t n = gdem_num_particles(h);
  std::vector<double> x(3 * n), v(3 * n), om(3 * n);
  std::vector<int> coord(n), cls(n);
  check(gdem_download_state(h, x.data(), v.data(), om.data(), nullptr, nullptr, nullptr,
                            nullptr));
  check(gdem_download_coordination(h, coord.data()));
  check(gdem_download_classes(h, cls.data()));
  const double* src[9] = {x.data(), x.data() + 1, x.data() + 2, v.data(), v.data() + 1,
                          v.data() + 2, om.data(), om.data() + 1, om.data() + 2};
  const std::string type_name = w.root + "_particleType.dat";
  FILE* ft = std::fopen(type_name.c_str(), w.binary ? "wb" : "w");
  if (!ft) throw std::runtime_error("cannot open " + type_name);
  try {
    if (w.binary) {
      std::vector<double> col(n);
      for (int k = 0; k < 9; ++k) {
        put(w.f[k], &time, sizeof time, w.root + kSuffix[k]);
        // the reference writes the time into the last file twice (:170-181)
        if (k == 8) put(w.f[k], &time, sizeof time, w.root + kSuffix[k]);
        for (int64_t i = 0; i < n; ++i) col[i] = src[k][3 * i];
        put(w.f[k], col.data(), n * sizeof(double), w.root + kSuffix[k]);
      }
      put(w.f[9], coord.data(), n * sizeof(int), w.root + kSuffix[9]);
      put(ft, cls.data(), n * sizeof(int), type_name);
    } else {
      std::string line, stime;
      number(stime, time);
      line.reserve((size_t)n * 14 + 16);
      for (int k = 0; k < 9; ++k) {
        line = stime;
        for (int64_t i = 0; i < n; ++i) {
          line += ' ';
          number(line, src[k][3 * i]);
        }
        line += '\n';
        put(w.f[k], line.data(), line.size(), w.root + kSuffix[k]);
      }
      char buf[16];
      line.clear();
      for (int64_t i = 0; i < n; ++i) {
        std::snprintf(buf, sizeof buf, " %d", coord[i]);
        line += buf;
      }
      line += '\n';
      put(w.f[9], line.data(), line.size(), w.root + kSuffix[9]);
      line.clear();
      for (int64_t i = 0; i < n; ++i) {
        std::snprintf(buf, sizeof buf, "%d ", cls[i]);
        line += buf;
      }
      line += '\n';
      put(ft, line.data(), line.size(), type_name);
    }
    for (FILE* f : w.f) std::fflush(f);
  } catch (...) {
    std::fclose(ft);
    throw;
  }
  if (std::fclose(ft) != 0) throw std::runtime_error("cannot write " + type_name);
}

template <typename F>
int guardedIo(F&& f) {
  try {
    f();
    return GDEM_OK;
  } catch (std::exception const& e) {
    gdem::setLastError(e.what());
    return GDEM_ERR_INVALID;
  }
}

}  // namespace

extern "C" {

int gdem_rawdata_start(gdem_handle h, const char* root, int binary, int append, double time) {
  return guardedIo([&] {
    if (!h || !root) throw std::runtime_error("invalid arguments");
    // one system, not a batch of instances
    if (gdem_num_instances(h) != 1)
      throw std::runtime_error("a RawData writer covers one system, not a batch");
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_writers.find(h);
    if (it != g_writers.end()) {
      delete it->second;
      g_writers.erase(it);
    }
    RawWriter* w = new RawWriter();
    w->root = root;
    w->binary = binary != 0;
    const char* mode = append ? (w->binary ? "ab" : "a") : (w->binary ? "wb" : "w");
    try {
      for (int k = 0; k < 10; ++k) {
        const std::string name = w->root + kSuffix[k];
        w->f[k] = std::fopen(name.c_str(), mode);
        if (!w->f[k]) throw std::runtime_error("cannot open " + name);
      }
      writeTime(h, *w, time);
    } catch (...) {
      delete w;
      throw;
    }
    g_writers[h] = w;
  });
}

int gdem_rawdata_write(gdem_handle h, double time) {
  return guardedIo([&] {
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_writers.find(h);
    if (it == g_writers.end()) throw std::runtime_error("gdem_rawdata_start was not called");
    writeTime(h, *it->second, time);
  });
}

int gdem_rawdata_end(gdem_handle h) {
  return guardedIo([&] {
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_writers.find(h);
    if (it == g_writers.end()) return;
    delete it->second;
    g_writers.erase(it);
  });
}

int gdem_write_velocity_max_mean(gdem_handle h, const char* path, int append, double time) {
  return guardedIo([&] {
    if (!h || !path) throw std::runtime_error("invalid arguments");
    double vmax = 0., vmean = 0.;
    check(gdem_velocity_stats(h, &vmax, &vmean));
    std::string line;
    number(line, time);
    line += '\t';
    number(line, vmax);
    line += '\t';
    number(line, vmean);
    line += '\n';
    FILE* f = std::fopen(path, append ? "a" : "w");
    if (!f) throw std::runtime_error(std::string("cannot open ") + path);
    const bool ok = std::fwrite(line.data(), 1, line.size(), f) == line.size();
    if (std::fclose(f) != 0 || !ok) throw std::runtime_error(std::string("cannot write ") + path);
  });
}

}  // extern "C"
