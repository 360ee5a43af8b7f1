// host_io.cpp — scene file readers: Wavefront OBJ meshes and Radiance RGBE
// (.hdr) images.
//
// OBJ follows the reference loader parse_obj_file
// (nectar_render/csrc/hittable/include/hittable/mesh.h:39-141), which drives
// tinyobjloader with triangulation on: quads are split along the shorter
// diagonal and larger polygons are fanned (tinyobjloader ear-clips those),
// vertices are deduplicated on the (v, vt, vn) index triple in order of first
// use, missing normals become the normalised sum of face normals (or +y when
// that sum is zero), and per-vertex tangents are the orthogonalised sum of
// per-face uv-gradient tangents ((1,0,0) for faces with degenerate uvs).
//
// HDR implements the Radiance picture format (G. Ward, "Real Pixels",
// Graphics Gems II; the RGBE encoding with flat or new-style run-length
// scanlines), decoding a texel (r, g, b, e) with e != 0 to m * 2^(e - 136) for
// each mantissa m, and to 0 when e == 0: the conversion stbi_loadf performs
// for the reference (nectar_render/csrc/material/include/material/texture.h:28-47).
#include "host_io.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <algorithm>
#include <atomic>
#include <thread>
#include <unordered_map>

namespace nr {

namespace {

struct Key {
  int v, vt, vn;
  bool operator==(const Key& o) const { return v == o.v && vt == o.vt && vn == o.vn; }
};
struct KeyHash {
  size_t operator()(const Key& k) const {
    size_t h = std::hash<int>()(k.v);
    h = h * 1000003u ^ std::hash<int>()(k.vt);
    h = h * 1000003u ^ std::hash<int>()(k.vn);
    return h;
  }
};

// host vector helpers with the reference's operation order
struct H3 {
  float x, y, z;
};
inline H3 sub(H3 a, H3 b) { return H3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline H3 add(H3 a, H3 b) { return H3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline H3 muls(H3 a, float t) { return H3{a.x * t, a.y * t, a.z * t}; }
inline float lsq(H3 v) {
  float o = v.x * v.x + v.y * v.y;
  o += v.z * v.z;
  return o;
}
inline float len(H3 v) { return sqrtf(lsq(v)); }
inline H3 nrm(H3 v) {
  float r = 1.0f / len(v);
  return H3{v.x * r, v.y * r, v.z * r};
}
inline H3 crs(H3 u, H3 v) {
  return H3{u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x};
}
inline float dt(H3 u, H3 v) { return u.x * v.x + u.y * v.y + u.z * v.z; }

// OBJ index: 1-based, negative = relative to the end
int resolve(long idx, size_t count) {
  if (idx > 0) return (int)(idx - 1);
  if (idx < 0) return (int)((long)count + idx);
  return -1;
}

}  // namespace

namespace {
struct Corner {
  int v, vt, vn;
};
static_assert(sizeof(Corner) == 3 * sizeof(int32_t), "corners are stored as int triples");
}  // namespace

namespace {

enum LineKind { kOther, kV, kVN, kVT, kF };

// The kind of an OBJ line (leading blanks skipped) and where its data starts.
LineKind classify(const char*& s) {
  while (*s == ' ' || *s == '\t') ++s;
  if (s[0] == 'v' && (s[1] == ' ' || s[1] == '\t')) return kV;
  if (s[0] == 'v' && s[1] == 'n' && (s[2] == ' ' || s[2] == '\t')) return kVN;
  if (s[0] == 'v' && s[1] == 't' && (s[2] == ' ' || s[2] == '\t')) return kVT;
  if (s[0] == 'f' && (s[1] == ' ' || s[1] == '\t')) return kF;
  return kOther;
}

// Calls fn(line, number) for every line of [begin, end) (split at '\n', as
// std::getline does), each copied into a NUL-terminated buffer so that the
// number parsers stop at its end.
template <typename F>
void for_lines(const char* begin, const char* end, size_t first_lineno, F&& fn) {
  std::string line;
  size_t lineno = first_lineno;
  for (const char* p = begin; p < end;) {
    const char* q = static_cast<const char*>(memchr(p, '\n', (size_t)(end - p)));
    if (!q) q = end;
    line.assign(p, (size_t)(q - p));
    fn(line.c_str(), ++lineno);
    p = q + 1;
  }
}

struct ChunkCounts {
  size_t lines = 0, v = 0, vn = 0, vt = 0;
};

}  // namespace

// The file is read whole and cut at line ends into chunks that the host
// threads take in turn. Pass 1 counts each chunk's lines and v / vn /
// vt records; pass 2 parses the v / vn / vt records into their final places;
// pass 3 parses the faces, resolving indices against the counts of records
// before the face's line (a prefix over the chunks). The result and the
// first error reported are those of reading the lines in order.
bool parse_obj(const std::string& path, ObjRaw& raw, std::string& err) {
  std::string data;
  {
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) {
      err = "Failed to load OBJ '" + path + "': cannot open file";
      return false;
    }
    fseek(f, 0, SEEK_END);
    const long len = ftell(f);
    fseek(f, 0, SEEK_SET);
    data.resize(len > 0 ? (size_t)len : 0);
    const size_t got = data.empty() ? 0 : fread(&data[0], 1, data.size(), f);
    fclose(f);
    data.resize(got);
  }
  const char* base = data.data();
  const size_t size = data.size();
  // chunks of >= 256 KB, several per thread, taken by the threads in turn
  // (the records of an OBJ file come in long runs of one kind)
  const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nch = std::max<size_t>(1, std::min<size_t>({8 * hw, 1024, size >> 18}));
  const size_t nthreads = std::min(hw, nch);
  std::vector<size_t> cut(nch + 1, size);
  cut[0] = 0;
  for (size_t k = 1; k < nch; ++k) {
    size_t at = std::max(cut[k - 1], size * k / nch);
    const void* nl = at < size ? memchr(base + at, '\n', size - at) : nullptr;
    cut[k] = nl ? (size_t)(static_cast<const char*>(nl) - base) + 1 : size;
  }
  auto run = [&](auto&& job) {
    std::atomic<size_t> next{0};
    auto worker = [&]() {
      for (size_t k; (k = next.fetch_add(1)) < nch;) job(k);
    };
    std::vector<std::thread> pool;
    for (size_t t = 1; t < nthreads; ++t) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
  };
  // pass 1: counts
  std::vector<ChunkCounts> cnt(nch);
  run([&](size_t k) {
    ChunkCounts& c = cnt[k];
    for_lines(base + cut[k], base + cut[k + 1], 0, [&](const char* s, size_t) {
      ++c.lines;
      switch (classify(s)) {
        case kV: ++c.v; break;
        case kVN: ++c.vn; break;
        case kVT: ++c.vt; break;
        default: break;
      }
    });
  });
  std::vector<ChunkCounts> pre(nch);
  for (size_t k = 1; k < nch; ++k) {
    pre[k].lines = pre[k - 1].lines + cnt[k - 1].lines;
    pre[k].v = pre[k - 1].v + cnt[k - 1].v;
    pre[k].vn = pre[k - 1].vn + cnt[k - 1].vn;
    pre[k].vt = pre[k - 1].vt + cnt[k - 1].vt;
  }
  const ChunkCounts& last = pre[nch - 1];
  std::vector<float>& vpos = raw.vpos;
  std::vector<float>& vnor = raw.vnor;
  std::vector<float>& vtex = raw.vtex;
  vpos.assign(3 * (last.v + cnt[nch - 1].v), 0.0f);
  vnor.assign(3 * (last.vn + cnt[nch - 1].vn), 0.0f);
  vtex.assign(2 * (last.vt + cnt[nch - 1].vt), 0.0f);
  // pass 2: vertex records
  run([&](size_t k) {
    size_t iv = pre[k].v, in = pre[k].vn, it = pre[k].vt;
    for_lines(base + cut[k], base + cut[k + 1], 0, [&](const char* s, size_t) {
      char* e;
      switch (classify(s)) {
        case kV: {
          const float a = strtof(s + 2, &e), b = strtof(e, &e), c = strtof(e, &e);
          vpos[3 * iv] = a;
          vpos[3 * iv + 1] = b;
          vpos[3 * iv + 2] = c;
          ++iv;
          break;
        }
        case kVN: {
          const float a = strtof(s + 3, &e), b = strtof(e, &e), c = strtof(e, &e);
          vnor[3 * in] = a;
          vnor[3 * in + 1] = b;
          vnor[3 * in + 2] = c;
          ++in;
          break;
        }
        case kVT: {
          const float a = strtof(s + 3, &e), b = strtof(e, &e);
          vtex[2 * it] = a;
          vtex[2 * it + 1] = b;
          ++it;
          break;
        }
        default: break;
      }
    });
  });
  // pass 3: faces
  std::vector<std::vector<Corner>> tris_k(nch);
  std::vector<std::string> err_k(nch);
  run([&](size_t k) {
    size_t nv = pre[k].v, nn = pre[k].vn, nt = pre[k].vt;  // records before the line
    std::vector<Corner>& tris = tris_k[k];
    std::vector<Corner> poly;
    bool bad = false;
    for_lines(base + cut[k], base + cut[k + 1], pre[k].lines, [&](const char* s, size_t lineno) {
      if (bad) return;
      switch (classify(s)) {
        case kV: ++nv; return;
        case kVN: ++nn; return;
        case kVT: ++nt; return;
        case kF: break;
        default: return;
      }
      poly.clear();
      const char* p = s + 2;
      while (*p) {
        while (*p == ' ' || *p == '\t') ++p;
        if (!*p || *p == '\r' || *p == '#') break;
        char* e;
        long vi = strtol(p, &e, 10), ti = 0, ni = 0;
        if (e == p) {
          err_k[k] = "Failed to load OBJ '" + path + "': bad face at line " + std::to_string(lineno);
          bad = true;
          return;
        }
        p = e;
        if (*p == '/') {
          ++p;
          if (*p != '/') {
            ti = strtol(p, &e, 10);
            p = e;
          }
          if (*p == '/') {
            ++p;
            ni = strtol(p, &e, 10);
            p = e;
          }
        }
        Corner c{resolve(vi, nv), ti ? resolve(ti, nt) : -1, ni ? resolve(ni, nn) : -1};
        if (c.v < 0 || (size_t)c.v >= nv) {
          err_k[k] = "Failed to load OBJ '" + path + "': vertex index out of range at line " +
                     std::to_string(lineno);
          bad = true;
          return;
        }
        if ((ti && (c.vt < 0 || (size_t)c.vt >= nt)) || (ni && (c.vn < 0 || (size_t)c.vn >= nn))) {
          err_k[k] = "Failed to load OBJ '" + path + "': texture or normal index out of range at line " +
                     std::to_string(lineno);
          bad = true;
          return;
        }
        poly.push_back(c);
        while (*p && *p != ' ' && *p != '\t') ++p;
      }
      if (poly.size() == 4) {
        // quads split along the shorter diagonal, as tinyobjloader does
        auto coord = [&](int v, int kk) { return vpos[3 * (size_t)v + kk]; };
        float e02x = coord(poly[2].v, 0) - coord(poly[0].v, 0);
        float e02y = coord(poly[2].v, 1) - coord(poly[0].v, 1);
        float e02z = coord(poly[2].v, 2) - coord(poly[0].v, 2);
        float e13x = coord(poly[3].v, 0) - coord(poly[1].v, 0);
        float e13y = coord(poly[3].v, 1) - coord(poly[1].v, 1);
        float e13z = coord(poly[3].v, 2) - coord(poly[1].v, 2);
        float s02 = e02x * e02x + e02y * e02y + e02z * e02z;
        float s13 = e13x * e13x + e13y * e13y + e13z * e13z;
        const int a[6] = {0, 1, 2, 0, 2, 3}, b[6] = {0, 1, 3, 1, 2, 3};
        for (int j = 0; j < 6; ++j) tris.push_back(poly[s02 < s13 ? a[j] : b[j]]);
      } else {
        // larger polygons are fanned (tinyobjloader ear-clips them)
        for (size_t j = 2; j < poly.size(); ++j) {
          tris.push_back(poly[0]);
          tris.push_back(poly[j - 1]);
          tris.push_back(poly[j]);
        }
      }
    });
  });
  for (size_t k = 0; k < nch; ++k)
    if (!err_k[k].empty()) {
      err = err_k[k];
      return false;
    }
  size_t total = 0;
  for (auto& t : tris_k) total += t.size();
  raw.corners.resize(3 * total);
  size_t at = 0;
  for (auto& t : tris_k) {
    std::memcpy(raw.corners.data() + 3 * at, t.data(), t.size() * sizeof(Corner));
    at += t.size();
  }
  return true;
}

void assemble_obj(const ObjRaw& raw, HostMesh& out) {
  const std::vector<float>& vpos = raw.vpos;
  const std::vector<float>& vnor = raw.vnor;
  const std::vector<float>& vtex = raw.vtex;
  const Corner* tris_p = reinterpret_cast<const Corner*>(raw.corners.data());
  const size_t n_corners = raw.corners.size() / 3;
  bool has_normals = !vnor.empty();
  out = HostMesh{};
  std::unordered_map<Key, uint32_t, KeyHash> uniq;
  uniq.reserve(n_corners);
  std::vector<H3> P, N, T;
  std::vector<float> UV;
  out.triangles.reserve(n_corners);
  for (size_t i = 0; i < n_corners; ++i) {
    const Corner& c = tris_p[i];
    Key k{c.v, c.vt, c.vn};
    auto it = uniq.find(k);
    if (it != uniq.end()) {
      out.triangles.push_back(it->second);
      continue;
    }
    uint32_t id = (uint32_t)P.size();
    P.push_back(H3{vpos[3 * c.v], vpos[3 * c.v + 1], vpos[3 * c.v + 2]});
    N.push_back(c.vn >= 0 ? H3{vnor[3 * c.vn], vnor[3 * c.vn + 1], vnor[3 * c.vn + 2]}
                          : H3{0.f, 0.f, 0.f});
    UV.push_back(c.vt >= 0 ? vtex[2 * c.vt] : 0.0f);
    UV.push_back(c.vt >= 0 ? vtex[2 * c.vt + 1] : 0.0f);
    T.push_back(H3{0.f, 0.f, 0.f});
    uniq.emplace(k, id);
    out.triangles.push_back(id);
  }
  size_t nt = out.triangles.size() / 3;
  const uint32_t* tr = out.triangles.data();
  if (!has_normals) {
    for (size_t t = 0; t < nt; ++t) {
      uint32_t a = tr[3 * t], b = tr[3 * t + 1], c = tr[3 * t + 2];
      H3 fn = nrm(crs(sub(P[b], P[a]), sub(P[c], P[a])));
      N[a] = add(N[a], fn);
      N[b] = add(N[b], fn);
      N[c] = add(N[c], fn);
    }
    for (auto& n : N) n = len(n) < 1e-8f ? H3{0.f, 1.f, 0.f} : nrm(n);
  }
  for (size_t t = 0; t < nt; ++t) {
    uint32_t a = tr[3 * t], b = tr[3 * t + 1], c = tr[3 * t + 2];
    H3 e1 = sub(P[b], P[a]), e2 = sub(P[c], P[a]);
    float du1 = UV[2 * b] - UV[2 * a], dv1 = UV[2 * b + 1] - UV[2 * a + 1];
    float du2 = UV[2 * c] - UV[2 * a], dv2 = UV[2 * c + 1] - UV[2 * a + 1];
    float denom = du1 * dv2 - du2 * dv1;
    H3 tg = fabsf(denom) < 1e-8f ? H3{1.f, 0.f, 0.f}
                                 : muls(sub(muls(e1, dv2), muls(e2, dv1)), 1.0f / denom);
    T[a] = add(T[a], tg);
    T[b] = add(T[b], tg);
    T[c] = add(T[c], tg);
  }
  for (size_t i = 0; i < T.size(); ++i) {
    H3 t = sub(T[i], muls(N[i], dt(T[i], N[i])));
    T[i] = len(t) < 1e-8f ? H3{1.f, 0.f, 0.f} : nrm(t);
  }
  size_t nv = P.size();
  out.positions.resize(3 * nv);
  out.normals.resize(3 * nv);
  out.tangents.resize(3 * nv);
  out.uvs = UV;
  for (size_t i = 0; i < nv; ++i) {
    out.positions[3 * i] = P[i].x;
    out.positions[3 * i + 1] = P[i].y;
    out.positions[3 * i + 2] = P[i].z;
    out.normals[3 * i] = N[i].x;
    out.normals[3 * i + 1] = N[i].y;
    out.normals[3 * i + 2] = N[i].z;
    out.tangents[3 * i] = T[i].x;
    out.tangents[3 * i + 1] = T[i].y;
    out.tangents[3 * i + 2] = T[i].z;
  }
}

bool load_obj(const std::string& path, HostMesh& out, std::string& err) {
  ObjRaw raw;
  if (!parse_obj(path, raw, err)) return false;
  assemble_obj(raw, out);
  return true;
}

namespace {
inline void rgbe_to_float(const uint8_t* in, float* out) {
  if (in[3] != 0) {
    float f = (float)ldexp(1.0f, (int)in[3] - (int)(128 + 8));
    out[0] = in[0] * f;
    out[1] = in[1] * f;
    out[2] = in[2] * f;
  } else {
    out[0] = out[1] = out[2] = 0.0f;
  }
}
}  // namespace

bool load_hdr(const std::string& path, HostImageF& out, std::string& err) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) {
    err = "Failed to load HDRI: cannot open '" + path + "'";
    return false;
  }
  std::vector<uint8_t> data;
  {
    uint8_t buf[1 << 16];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), f)) > 0) data.insert(data.end(), buf, buf + n);
    fclose(f);
  }
  size_t pos = 0;
  auto read_line = [&](std::string& l) {
    l.clear();
    while (pos < data.size() && data[pos] != '\n') l.push_back((char)data[pos++]);
    if (pos < data.size()) ++pos;
    return true;
  };
  std::string l;
  read_line(l);
  if (l != "#?RADIANCE" && l != "#?RGBE") {
    err = "Failed to load HDRI: not a Radiance file";
    return false;
  }
  bool fmt_ok = false;
  while (pos < data.size()) {
    read_line(l);
    if (l.empty()) break;
    if (l == "FORMAT=32-bit_rle_rgbe") fmt_ok = true;
  }
  if (!fmt_ok) {
    err = "Failed to load HDRI: unsupported format";
    return false;
  }
  read_line(l);
  int H = 0, W = 0;
  if (sscanf(l.c_str(), "-Y %d +X %d", &H, &W) != 2 || H <= 0 || W <= 0) {
    err = "Failed to load HDRI: unsupported image orientation";
    return false;
  }
  out.C = 3;
  out.H = (uint32_t)H;
  out.W = (uint32_t)W;
  std::vector<float> hwc((size_t)H * W * 3);
  std::vector<uint8_t> scan((size_t)W * 4);
  for (int y = 0; y < H; ++y) {
    if (pos + 4 > data.size()) {
      err = "Failed to load HDRI: truncated file";
      return false;
    }
    bool rle = W >= 8 && W < 32768 && data[pos] == 2 && data[pos + 1] == 2 &&
               !(data[pos + 2] & 0x80) && (((int)data[pos + 2] << 8) | data[pos + 3]) == W;
    if (!rle) {
      // flat scanlines for the whole remaining image
      size_t need = (size_t)(H - y) * W * 4;
      if (pos + need > data.size()) {
        err = "Failed to load HDRI: truncated file";
        return false;
      }
      for (; y < H; ++y)
        for (int x = 0; x < W; ++x, pos += 4) rgbe_to_float(&data[pos], &hwc[((size_t)y * W + x) * 3]);
      break;
    }
    pos += 4;
    for (int ch = 0; ch < 4; ++ch) {
      int x = 0;
      while (x < W) {
        if (pos >= data.size()) {
          err = "Failed to load HDRI: truncated file";
          return false;
        }
        int count = data[pos++];
        if (count > 128) {
          count -= 128;
          if (count > W - x || pos >= data.size()) {
            err = "Failed to load HDRI: bad run";
            return false;
          }
          uint8_t v = data[pos++];
          for (int k = 0; k < count; ++k) scan[(size_t)(x++) * 4 + ch] = v;
        } else {
          if (count == 0 || count > W - x || pos + count > data.size()) {
            err = "Failed to load HDRI: bad dump";
            return false;
          }
          for (int k = 0; k < count; ++k) scan[(size_t)(x++) * 4 + ch] = data[pos++];
        }
      }
    }
    for (int x = 0; x < W; ++x) rgbe_to_float(&scan[(size_t)x * 4], &hwc[((size_t)y * W + x) * 3]);
  }
  // planar CHW, as the reference's load_image_float (texture.h:28-47)
  size_t hw = (size_t)H * W;
  out.chw.resize(hw * 3);
  for (size_t c = 0; c < 3; ++c)
    for (size_t i = 0; i < hw; ++i) out.chw[c * hw + i] = hwc[i * 3 + c];
  return true;
}

}  // namespace nr
