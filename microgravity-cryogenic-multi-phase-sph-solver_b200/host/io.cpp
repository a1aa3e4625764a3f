// io.cpp -- the two output formats of the reference (io.hpp:13-22): legacy
// binary VTK polydata and the viewer's JSON frame.
//
// Both writers here take a packed payload and add only the text around it:
//   * VTK: the payload is the file's binary data as big-endian 32-bit words,
//     section after section (POINTS, VERTICES, the scalars, VECTORS).  The
//     solver has the device write it (cryo_frame_vtk); for host particles
//     the same layout is packed here.  The writer walks a section table.
//   * JSON: the payload is the viewer frame's arrays, walls already dropped
//     if asked (the device compacts them, cryo_frame_viewer; host frames are
//     filtered here).  Numbers are formatted with std::to_chars into one
//     buffer that is written with a single call.
// The file layouts (header lines, section order, the JSON keys and their
// number formats: %.9g time, %.6g values, non-finite values written as 0)
// are the reference's, so files from either build read the same.
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "cryosph.hpp"

namespace cryosph {

namespace {

struct FileDeleter {
  void operator()(std::FILE* f) const noexcept {
    if (f) std::fclose(f);
  }
};
using File = std::unique_ptr<std::FILE, FileDeleter>;

File open_or_throw(const std::string& path, const char* who) {
  File f(std::fopen(path.c_str(), "wb"));
  if (!f) throw std::runtime_error(std::string(who) + ": cannot open '" + path + "'");
  return f;
}

std::uint32_t swap_bytes(std::uint32_t w) {
  return (w >> 24) | ((w >> 8) & 0xff00u) | ((w << 8) & 0xff0000u) | (w << 24);
}
std::uint32_t big_endian_word(float f) {
  std::uint32_t w;
  std::memcpy(&w, &f, 4);
  return swap_bytes(w);
}

// Text before each binary section of the VTK file and the section's size in
// words per particle (the payload holds the sections in this order).
struct VtkSection {
  std::string head;
  std::size_t words;
};

std::vector<VtkSection> vtk_sections(std::size_t n, bool with_pressure) {
  const std::string N = std::to_string(n);
  auto scalar = [](const char* name) {
    return std::string("SCALARS ") + name + " float 1\nLOOKUP_TABLE default\n";
  };
  std::vector<VtkSection> s;
  s.push_back({"# vtk DataFile Version 3.0\nCryoSPH-CUDA particles\nBINARY\nDATASET POLYDATA\nPOINTS " + N +
                   " float\n",
               3});
  s.push_back({"\nVERTICES " + N + " " + std::to_string(2 * n) + "\n", 2});
  s.push_back({"\nPOINT_DATA " + N + "\n" + scalar("temperature"), 1});
  for (const char* name : {"mass", "density", "phase"}) s.push_back({"\n" + scalar(name), 1});
  if (with_pressure) s.push_back({"\n" + scalar("pressure"), 1});
  s.push_back({"\nVECTORS velocity float\n", 3});
  return s;
}

void write_vtk_payload(const std::string& path, std::size_t n, const std::uint32_t* words, bool with_pressure) {
  File f = open_or_throw(path, "write_vtk");
  const std::uint32_t* at = words;
  for (const VtkSection& sec : vtk_sections(n, with_pressure)) {
    std::fwrite(sec.head.data(), 1, sec.head.size(), f.get());
    if (n) std::fwrite(at, 4, sec.words * n, f.get());
    at += sec.words * n;
  }
  std::fputc('\n', f.get());
  if (std::ferror(f.get())) throw std::runtime_error("write_vtk: write failed for '" + path + "'");
}

// JSON number formatting into a growing buffer.
class JsonOut {
 public:
  explicit JsonOut(std::size_t reserve) { buf_.reserve(reserve); }
  JsonOut& raw(const char* s) {
    buf_.append(s);
    return *this;
  }
  JsonOut& num(double v, int precision) {
    char tmp[40];
    const auto r = std::to_chars(tmp, tmp + sizeof tmp, v, std::chars_format::general, precision);
    buf_.append(tmp, r.ptr);
    return *this;
  }
  JsonOut& integer(long long v) {
    char tmp[24];
    const auto r = std::to_chars(tmp, tmp + sizeof tmp, v);
    buf_.append(tmp, r.ptr);
    return *this;
  }
  // "key":[v0,v1,...] of float values (non-finite ones as 0)
  JsonOut& floats(const char* key, const float* v, std::size_t count, std::size_t stride = 1) {
    raw(",\"").raw(key).raw("\":[");
    for (std::size_t k = 0; k < count; ++k) {
      if (k) buf_.push_back(',');
      const float x = v[k * stride];
      num(std::isfinite(x) ? static_cast<double>(x) : 0.0, 6);
    }
    buf_.push_back(']');
    return *this;
  }
  const std::string& str() const { return buf_; }

 private:
  std::string buf_;
};

// The viewer frame file from packed arrays of `count` particles.
void write_viewer_json(const std::string& path, double time, long long step, std::size_t count, const float* position,
                       const std::uint8_t* phase, const float* temperature, const float* pressure, const float* speed) {
  JsonOut j(64 + count * 64);
  j.raw("{\"time\":").num(time, 9).raw(",\"step\":").integer(step).raw(",\"n\":").integer(static_cast<long long>(count));
  j.raw(",\"position\":[");
  for (std::size_t k = 0; k < 3 * count; ++k) {
    if (k) j.raw(",");
    j.num(static_cast<double>(position[k]), 6);
  }
  j.raw("],\"phase\":[");
  for (std::size_t k = 0; k < count; ++k) {
    if (k) j.raw(",");
    j.integer(phase[k]);
  }
  j.raw("]");
  j.floats("temperature", temperature, count).floats("pressure", pressure, count).floats("speed", speed, count);
  j.raw("}\n");
  File f = open_or_throw(path, "write_json_frame");
  std::fwrite(j.str().data(), 1, j.str().size(), f.get());
  if (std::ferror(f.get())) throw std::runtime_error("write_json_frame: write failed for '" + path + "'");
}

}  // namespace

// Host particles into the VTK payload layout (the device path packs the same
// words in cryo_frame_vtk).
void write_vtk(const std::string& path, const HostParticles& hp, const std::vector<real>& pressure) {
  const std::size_t n = hp.size();
  const bool with_p = pressure.size() == n;
  std::vector<std::uint32_t> w((with_p ? CRYO_VTK_WORDS_PER_PARTICLE : CRYO_VTK_WORDS_PER_PARTICLE - 1) * n);
  std::uint32_t* o = w.data();
  auto vec_section = [&](const std::vector<Vec3>& v) {
    for (const Vec3& a : v) {
      *o++ = big_endian_word(a.x);
      *o++ = big_endian_word(a.y);
      *o++ = big_endian_word(a.z);
    }
  };
  vec_section(hp.x);
  for (std::size_t i = 0; i < n; ++i) {
    *o++ = swap_bytes(1u);
    *o++ = swap_bytes(static_cast<std::uint32_t>(i));
  }
  for (const std::vector<real>* col : {&hp.T, &hp.m, &hp.rho})
    for (real a : *col) *o++ = big_endian_word(a);
  for (std::uint8_t ph : hp.phase) *o++ = big_endian_word(static_cast<float>(ph));
  if (with_p)
    for (real a : pressure) *o++ = big_endian_word(a);
  vec_section(hp.v);
  write_vtk_payload(path, n, w.data(), with_p);
}

TelemetryFrame make_frame(const HostParticles& hp, const std::vector<real>& pressure, double time, long long step) {
  const std::size_t n = hp.size();
  TelemetryFrame f;
  f.time = time;
  f.step = step;
  f.n = static_cast<int>(n);
  f.position.assign(reinterpret_cast<const float*>(hp.x.data()), reinterpret_cast<const float*>(hp.x.data()) + 3 * n);
  f.temperature = hp.T;
  f.pressure = pressure.size() == n ? pressure : std::vector<real>(n, real(0));
  f.speed.resize(n);
  for (std::size_t i = 0; i < n; ++i) f.speed[i] = norm(hp.v[i]);
  f.phase = hp.phase;
  return f;
}

void write_json_frame(const std::string& path, const TelemetryFrame& fr, bool include_walls) {
  const std::size_t n = static_cast<std::size_t>(fr.n);
  if (include_walls) {
    write_viewer_json(path, fr.time, fr.step, n, fr.position.data(), fr.phase.data(), fr.temperature.data(),
                      fr.pressure.data(), fr.speed.data());
    return;
  }
  std::vector<float> pos, T, p, s;
  std::vector<std::uint8_t> ph;
  for (std::size_t i = 0; i < n; ++i) {
    if (fr.phase[i] == kWall) continue;
    pos.insert(pos.end(), fr.position.begin() + 3 * i, fr.position.begin() + 3 * i + 3);
    T.push_back(fr.temperature[i]);
    p.push_back(fr.pressure[i]);
    s.push_back(fr.speed[i]);
    ph.push_back(fr.phase[i]);
  }
  write_viewer_json(path, fr.time, fr.step, ph.size(), pos.data(), ph.data(), T.data(), p.data(), s.data());
}

// Solver::write_vtk / write_json: the device packs the payload.
void Solver::write_vtk(const std::string& path) const {
  int n = 0;
  check(cryo_frame_vtk(ctx_, nullptr, 0, &n));
  std::vector<std::uint32_t> w(static_cast<std::size_t>(n) * CRYO_VTK_WORDS_PER_PARTICLE);
  check(cryo_frame_vtk(ctx_, w.data(), w.size() * 4, &n));
  write_vtk_payload(path, static_cast<std::size_t>(n), w.data(), true);
}

void Solver::write_json(const std::string& path, bool include_walls) const {
  const std::size_t n = num_particles();
  std::vector<float> pos(3 * n), T(n), p(n), s(n);
  std::vector<std::uint8_t> ph(n);
  int count = 0;
  check(cryo_frame_viewer(ctx_, include_walls ? 1 : 0, pos.data(), T.data(), p.data(), s.data(), ph.data(),
                          static_cast<int>(n), &count));
  write_viewer_json(path, time(), step_count(), static_cast<std::size_t>(count), pos.data(), ph.data(), T.data(),
                    p.data(), s.data());
}

}  // namespace cryosph
