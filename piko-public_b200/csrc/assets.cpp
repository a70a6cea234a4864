// Scene and mesh loaders without GL: the reference's `.scene` command files
// (pikoc/samples/rasterPipelineFixPt/sceneParser/sceneParser.cpp:114-478), its
// bezmesh `.dat` reader (bezmesh/bezmesh.cpp:23-80,130-150) and Wavefront OBJ
// meshes in place of assimp (whose library is not shipped), flattened the way
// scene::flatten does (basicTypes/scene.h:134-190) into the per-vertex-slot
// arrays a PIKO_SCENE_TRIANGLES / PIKO_SCENE_PATCHES descriptor takes.
//
// The reference keeps its model transform on the GL matrix stack
// (glTranslatef / glRotatef / glScalef, each post-multiplying the current
// matrix) and reads it back as floats.  Here the same products are formed on
// the CPU in double precision and every transformed value is rounded to float
// once; the GL driver's own float rounding is not reproducible, so positions of
// a loaded scene can differ from the reference's by an ulp.  Camera matrices
// follow camera::updateCam (basicTypes/camera.h:73-120).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/piko_b200.h"

namespace {

using Mat = std::array<double, 16>;  // column-major, as GL stores it
constexpr double kPi = 3.14159265358979323846;

Mat identity()
{
  Mat m{};
  m[0] = m[5] = m[10] = m[15] = 1.0;
  return m;
}

Mat mul(const Mat& a, const Mat& b)
{
  Mat r{};
  for (int c = 0; c < 4; ++c)
    for (int rr = 0; rr < 4; ++rr) {
      double s = 0.0;
      for (int k = 0; k < 4; ++k) s += a[k * 4 + rr] * b[c * 4 + k];
      r[c * 4 + rr] = s;
    }
  return r;
}

Mat translate(double x, double y, double z)
{
  Mat m = identity();
  m[12] = x; m[13] = y; m[14] = z;
  return m;
}

Mat scale(double x, double y, double z)
{
  Mat m = identity();
  m[0] = x; m[5] = y; m[10] = z;
  return m;
}

// rotation by `deg` degrees about the axis (x, y, z), as glRotatef defines it
Mat rotate(double deg, double x, double y, double z)
{
  const double len = std::sqrt(x * x + y * y + z * z);
  Mat m = identity();
  if (len == 0.0) return m;
  x /= len; y /= len; z /= len;
  const double a = deg * kPi / 180.0, c = std::cos(a), s = std::sin(a), t = 1.0 - c;
  m[0] = t * x * x + c;     m[4] = t * x * y - s * z; m[8] = t * x * z + s * y;
  m[1] = t * x * y + s * z; m[5] = t * y * y + c;     m[9] = t * y * z - s * x;
  m[2] = t * x * z - s * y; m[6] = t * y * z + s * x; m[10] = t * z * z + c;
  return m;
}

bool invert(const Mat& m, Mat& out)
{
  // Gauss-Jordan on the 4x4 (row index r, column index c: m[c * 4 + r])
  double a[4][8];
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      a[r][c] = m[c * 4 + r];
      a[r][c + 4] = r == c ? 1.0 : 0.0;
    }
  for (int col = 0; col < 4; ++col) {
    int piv = col;
    for (int r = col + 1; r < 4; ++r)
      if (std::fabs(a[r][col]) > std::fabs(a[piv][col])) piv = r;
    if (a[piv][col] == 0.0) return false;
    if (piv != col)
      for (int c = 0; c < 8; ++c) std::swap(a[piv][c], a[col][c]);
    const double d = a[col][col];
    for (int c = 0; c < 8; ++c) a[col][c] /= d;
    for (int r = 0; r < 4; ++r) {
      if (r == col) continue;
      const double f = a[r][col];
      if (f != 0.0)
        for (int c = 0; c < 8; ++c) a[r][c] -= f * a[col][c];
    }
  }
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) out[c * 4 + r] = a[r][c + 4];
  return true;
}

struct Vec3 { double x, y, z; };

struct Camera {
  Vec3 eye{0.0, 0.0, 3.0}, target{0.0, 0.0, 0.0}, up{0.0, 1.0, 0.0};
  double fovy = kPi / 3.0, znear = 0.02, zfar = 100.0;   // camera.h:40-45 defaults
  bool set = false;
};

// One flattened triangle corner set: positions, normals (unit), uvs.
struct Tri {
  float p[3][3], n[3][3], t[3][2];
  float col[3];   // diffuse colour of its material
};

struct Asset {
  std::vector<Tri> tris;
  bool has_uv = false;
  std::vector<float> patches;   // [P][16][4]
  Camera cam;
  std::vector<std::array<float, 3>> lights;      // light positions, in file order
  std::vector<std::array<float, 3>> diffuse;     // material diffuse colours, in file order
};

thread_local std::string g_err;

piko_status fail(const std::string& msg)
{
  g_err = msg;
  return PIKO_ERR_INVALID;
}

// Tokens of a command file: '#' starts a comment, blanks and tabs separate
// tokens; commands and their arguments may span lines.
class Tokens {
 public:
  explicit Tokens(std::istream& in)
  {
    std::string line;
    while (std::getline(in, line)) {
      const size_t h = line.find('#');
      if (h != std::string::npos) line.resize(h);
      std::istringstream ls(line);
      std::string t;
      while (ls >> t) q_.push_back(t);
    }
  }
  bool empty() const { return q_.empty(); }
  const std::string& peek() const { return q_.front(); }
  bool next(std::string& t)
  {
    if (q_.empty()) return false;
    t = q_.front();
    q_.pop_front();
    return true;
  }
  bool num(double& v)
  {
    std::string t;
    if (!next(t)) return false;
    char* end = nullptr;
    v = std::strtod(t.c_str(), &end);
    return end && *end == '\0' && end != t.c_str();
  }
  // "[ a b ... ]" with n numbers
  bool vec(double* v, int n)
  {
    std::string t;
    if (!next(t) || t != "[") return false;
    for (int i = 0; i < n; ++i)
      if (!num(v[i])) return false;
    return next(t) && t == "]";
  }

 private:
  std::deque<std::string> q_;
};

std::string dirname_of(const std::string& p)
{
  const size_t s = p.find_last_of('/');
  return s == std::string::npos ? std::string(".") : p.substr(0, s);
}

std::string ext_of(const std::string& p)
{
  const size_t d = p.find_last_of('.');
  std::string e = d == std::string::npos ? std::string() : p.substr(d + 1);
  std::transform(e.begin(), e.end(), e.begin(), [](unsigned char c) { return (char)std::tolower(c); });
  return e;
}

// Wavefront OBJ: v, vn, vt, f (v, v/t, v//n, v/t/n; negative indices count
// from the end); polygons are split into fans.  A face without normals gets
// its geometric normal on all three corners.
piko_status load_obj(const std::string& path, const Mat& M, const float* col, Asset& A)
{
  std::ifstream in(path);
  if (!in) return fail("cannot open " + path);
  std::vector<std::array<double, 3>> V, N;
  std::vector<std::array<double, 2>> T;
  Mat inv;
  if (!invert(M, inv)) return fail("model transform is singular at " + path);
  std::string line;
  int lineno = 0;
  while (std::getline(in, line)) {
    ++lineno;
    const size_t h = line.find('#');
    if (h != std::string::npos) line.resize(h);
    std::istringstream ls(line);
    std::string kw;
    if (!(ls >> kw)) continue;
    if (kw == "v") {
      double x, y, z;
      if (!(ls >> x >> y >> z)) return fail(path + ":" + std::to_string(lineno) + ": bad vertex");
      V.push_back({x, y, z});
    } else if (kw == "vn") {
      double x, y, z;
      if (!(ls >> x >> y >> z)) return fail(path + ":" + std::to_string(lineno) + ": bad normal");
      N.push_back({x, y, z});
    } else if (kw == "vt") {
      double u, v = 0.0;
      if (!(ls >> u)) return fail(path + ":" + std::to_string(lineno) + ": bad texture coordinate");
      ls >> v;
      T.push_back({u, v});
    } else if (kw == "f") {
      std::vector<std::array<long, 3>> corners;   // v, t, n (0-based, -1 = absent)
      std::string c;
      while (ls >> c) {
        std::array<long, 3> ix{-1, -1, -1};
        size_t start = 0;
        for (int k = 0; k < 3; ++k) {
          const size_t sl = c.find('/', start);
          const std::string f = c.substr(start, sl == std::string::npos ? std::string::npos : sl - start);
          if (!f.empty()) {
            const long v = std::strtol(f.c_str(), nullptr, 10);
            const long n = k == 0 ? (long)V.size() : (k == 1 ? (long)T.size() : (long)N.size());
            const long i = v > 0 ? v - 1 : n + v;
            if (v == 0 || i < 0 || i >= n) return fail(path + ":" + std::to_string(lineno) + ": index out of range");
            ix[k] = i;
          }
          if (sl == std::string::npos) break;
          start = sl + 1;
        }
        if (ix[0] < 0) return fail(path + ":" + std::to_string(lineno) + ": face corner without a vertex");
        corners.push_back(ix);
      }
      if (corners.size() < 3) return fail(path + ":" + std::to_string(lineno) + ": face with fewer than 3 corners");
      for (size_t k = 1; k + 1 < corners.size(); ++k) {
        const std::array<long, 3>* cc[3] = {&corners[0], &corners[k], &corners[k + 1]};
        Tri t{};
        double wp[3][3];
        for (int q = 0; q < 3; ++q) {
          const auto& v = V[(*cc[q])[0]];
          for (int r = 0; r < 3; ++r) wp[q][r] = M[r] * v[0] + M[4 + r] * v[1] + M[8 + r] * v[2] + M[12 + r];
          for (int r = 0; r < 3; ++r) t.p[q][r] = (float)wp[q][r];
        }
        // geometric normal of the untransformed face, for corners without one
        const auto& a = V[(*cc[0])[0]];
        const auto& b = V[(*cc[1])[0]];
        const auto& d = V[(*cc[2])[0]];
        const double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
        const double e2[3] = {d[0] - a[0], d[1] - a[1], d[2] - a[2]};
        const double fn[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        for (int q = 0; q < 3; ++q) {
          double n[3] = {fn[0], fn[1], fn[2]};
          if ((*cc[q])[2] >= 0) {
            const auto& nn = N[(*cc[q])[2]];
            n[0] = nn[0]; n[1] = nn[1]; n[2] = nn[2];
          }
          // ntransform with the inverse model matrix, then unit length (scene.h:164-171)
          double tn[3];
          for (int r = 0; r < 3; ++r) tn[r] = n[0] * inv[r * 4 + 0] + n[1] * inv[r * 4 + 1] + n[2] * inv[r * 4 + 2];
          const double len = std::sqrt(tn[0] * tn[0] + tn[1] * tn[1] + tn[2] * tn[2]);
          for (int r = 0; r < 3; ++r) t.n[q][r] = (float)(len > 0.0 ? tn[r] / len : 0.0);
          if ((*cc[q])[1] >= 0) {
            t.t[q][0] = (float)T[(*cc[q])[1]][0];
            t.t[q][1] = (float)T[(*cc[q])[1]][1];
            A.has_uv = true;
          }
        }
        for (int r = 0; r < 3; ++r) t.col[r] = col[r];
        A.tris.push_back(t);
      }
    }
    // o, g, s, usemtl, mtllib and anything else: not needed for the pipeline
  }
  return PIKO_OK;
}

// The bezmesh reader: after every `Patch "bicubic"` line, 16 x y z points
// (w = 1); then all coordinates scaled by scale / maxcoord, maxcoord updated
// with the signed coordinate whenever its magnitude exceeds the current value
// (bezmesh.cpp:130-150); then the model transform.
piko_status load_bez(const std::string& path, double scale_factor, const Mat& M, Asset& A)
{
  std::ifstream in(path);
  if (!in) return fail("cannot open " + path);
  std::vector<float> cps;
  std::string line;
  std::vector<std::string> pending;
  bool in_patch = false;
  std::vector<float> cur;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    std::vector<std::string> tok;
    std::string t;
    while (ls >> t) tok.push_back(t);
    if (tok.size() >= 2 && tok[0] == "Patch" && tok[1] == "\"bicubic\"") {
      in_patch = true;
      cur.clear();
      continue;
    }
    if (!in_patch || tok.empty()) continue;
    for (const auto& s : tok) {
      char* end = nullptr;
      const float v = std::strtof(s.c_str(), &end);
      if (end == s.c_str()) return fail(path + ": bad control point value '" + s + "'");
      cur.push_back(v);
    }
    if (cur.size() >= 48) {
      for (int k = 0; k < 16; ++k) {
        cps.push_back(cur[3 * k]); cps.push_back(cur[3 * k + 1]); cps.push_back(cur[3 * k + 2]); cps.push_back(1.0f);
      }
      in_patch = false;
    }
  }
  if (scale_factor != 0.0 && !cps.empty()) {
    float maxcoord = 0.0f;
    for (size_t i = 0; i < cps.size(); i += 4)
      for (int c = 0; c < 3; ++c)
        if (std::fabs(cps[i + c]) > maxcoord) maxcoord = cps[i + c];
    const float factor = (float)scale_factor / maxcoord;
    for (size_t i = 0; i < cps.size(); i += 4)
      for (int c = 0; c < 3; ++c) cps[i + c] = cps[i + c] * factor;
  }
  for (size_t i = 0; i < cps.size(); i += 4) {
    const double x = cps[i], y = cps[i + 1], z = cps[i + 2], w = cps[i + 3];
    double o[4];
    for (int r = 0; r < 4; ++r) o[r] = M[r] * x + M[4 + r] * y + M[8 + r] * z + M[12 + r] * w;
    for (int r = 0; r < 4; ++r) A.patches.push_back((float)o[r]);
  }
  return PIKO_OK;
}

piko_status load_scene(const std::string& path, const std::string& mesh_dir, Asset& A)
{
  std::ifstream in(path);
  if (!in) return fail("cannot open " + path);
  Tokens tk(in);
  Mat M = identity();
  float curcol[3] = {0.9f, 0.9f, 0.6f};
  std::string cmd;
  while (tk.next(cmd)) {
    double v[12];
    if (cmd == "camera") {
      if (!tk.vec(v, 3) || !tk.vec(v + 3, 3) || !tk.vec(v + 6, 3)) return fail(path + ": bad camera");
      A.cam.eye = {v[0], v[1], v[2]};
      A.cam.target = {v[3], v[4], v[5]};
      A.cam.up = {v[6], v[7], v[8]};
      A.cam.fovy = kPi / 3.0;
      A.cam.set = true;
      // the optional aperture / focal length / focal plane triple (thin-lens
      // parameters; the rasterizers ignore them)
      if (!tk.empty() && tk.peek() == "[" && !tk.vec(v + 9, 3)) return fail(path + ": bad camera lens");
    } else if (cmd == "camera_fov") {
      if (!tk.num(v[0])) return fail(path + ": bad camera_fov");
      A.cam.fovy = v[0] * kPi / 180.0;
    } else if (cmd == "zNear") {
      if (!tk.num(v[0])) return fail(path + ": bad zNear");
      A.cam.znear = v[0];
    } else if (cmd == "zFar") {
      if (!tk.num(v[0])) return fail(path + ": bad zFar");
      A.cam.zfar = v[0];
    } else if (cmd == "light") {
      if (!tk.vec(v, 3) || !tk.vec(v + 3, 3) || !tk.vec(v + 6, 3) || !tk.num(v[9])) return fail(path + ": bad light");
      A.lights.push_back({(float)v[0], (float)v[1], (float)v[2]});
    } else if (cmd == "material") {
      if (!tk.vec(v, 3) || !tk.vec(v + 3, 3) || !tk.vec(v + 6, 3) || !tk.num(v[9])) return fail(path + ": bad material");
      curcol[0] = (float)v[3]; curcol[1] = (float)v[4]; curcol[2] = (float)v[5];
      A.diffuse.push_back({curcol[0], curcol[1], curcol[2]});
    } else if (cmd == "meshAttribute") {
      std::string name;
      if (!tk.next(name) || !tk.num(v[0])) return fail(path + ": bad meshAttribute");
    } else if (cmd == "translate") {
      if (!tk.vec(v, 3)) return fail(path + ": bad translate");
      M = mul(M, translate(v[0], v[1], v[2]));
    } else if (cmd == "rotate") {
      if (!tk.vec(v, 3) || !tk.num(v[3])) return fail(path + ": bad rotate");
      M = mul(M, rotate(v[3], v[0], v[1], v[2]));
    } else if (cmd == "scale") {
      if (!tk.vec(v, 3)) return fail(path + ": bad scale");
      M = mul(M, scale(v[0], v[1], v[2]));
    } else if (cmd == "reset") {
      M = identity();
    } else if (cmd == "texture") {
      std::string f;
      if (!tk.next(f)) return fail(path + ": bad texture");   // accepted and ignored, as the reference does
    } else if (cmd == "loadmesh") {
      std::string f;
      if (!tk.next(f)) return fail(path + ": bad loadmesh");
      const std::string mp = mesh_dir + "/" + f;
      if (ext_of(f) != "obj") return fail(mp + ": only OBJ meshes load here (the reference's assimp is not shipped)");
      const piko_status st = load_obj(mp, M, curcol, A);
      if (st != PIKO_OK) return st;
    } else if (cmd == "loadbez") {
      std::string f;
      if (!tk.next(f)) return fail(path + ": bad loadbez");
      const piko_status st = load_bez(mesh_dir + "/" + f, 1.0, M, A);
      if (st != PIKO_OK) return st;
    } else {
      return fail(path + ": unknown command '" + cmd + "'");
    }
  }
  return PIKO_OK;
}

// camera::updateCam (camera.h:73-120): a GL perspective matrix times a GL
// look-at matrix, column-major, rounded to float once.
void view_proj(const Camera& c, int W, int H, float* out)
{
  const double aspect = (double)W / (double)H;
  const double f = 1.0 / std::tan(c.fovy / 2.0), d = 1.0 / (c.znear - c.zfar);
  Mat P{};
  P[0] = f / aspect;
  P[5] = f;
  P[10] = (c.znear + c.zfar) * d;
  P[11] = -1.0;
  P[14] = 2.0 * c.znear * c.zfar * d;
  double fw[3] = {c.target.x - c.eye.x, c.target.y - c.eye.y, c.target.z - c.eye.z};
  double fl = std::sqrt(fw[0] * fw[0] + fw[1] * fw[1] + fw[2] * fw[2]);
  for (double& x : fw) x /= fl;
  double up[3] = {c.up.x, c.up.y, c.up.z};
  const double ul = std::sqrt(up[0] * up[0] + up[1] * up[1] + up[2] * up[2]);
  for (double& x : up) x /= ul;
  double s[3] = {fw[1] * up[2] - fw[2] * up[1], fw[2] * up[0] - fw[0] * up[2], fw[0] * up[1] - fw[1] * up[0]};
  const double sl = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
  for (double& x : s) x /= sl;
  const double u[3] = {s[1] * fw[2] - s[2] * fw[1], s[2] * fw[0] - s[0] * fw[2], s[0] * fw[1] - s[1] * fw[0]};
  Mat V = identity();
  for (int k = 0; k < 3; ++k) {
    V[k * 4 + 0] = s[k];
    V[k * 4 + 1] = u[k];
    V[k * 4 + 2] = -fw[k];
  }
  const double e[3] = {c.eye.x, c.eye.y, c.eye.z};
  V[12] = -(s[0] * e[0] + s[1] * e[1] + s[2] * e[2]);
  V[13] = -(u[0] * e[0] + u[1] * e[1] + u[2] * e[2]);
  V[14] = fw[0] * e[0] + fw[1] * e[1] + fw[2] * e[2];
  const Mat VP = mul(P, V);
  for (int i = 0; i < 16; ++i) out[i] = (float)VP[i];
}

}  // namespace

struct piko_asset {
  Asset a;
};

extern "C" {

const char* piko_asset_last_error(void) { return g_err.c_str(); }

piko_status piko_asset_load(const char* path, const char* mesh_dir, piko_asset** out)
{
  if (!path || !out) return fail("null argument");
  *out = nullptr;
  g_err.clear();
  const std::string p(path);
  const std::string md = mesh_dir ? std::string(mesh_dir) : dirname_of(p);
  piko_asset* as = new piko_asset();
  const std::string e = ext_of(p);
  piko_status st;
  const float ref_col[3] = {0.9f, 0.9f, 0.6f};
  if (e == "scene") st = load_scene(p, md, as->a);
  else if (e == "obj") st = load_obj(p, identity(), ref_col, as->a);
  else if (e == "dat") st = load_bez(p, 1.0, identity(), as->a);
  else st = fail(p + ": unknown file type (.scene, .obj or .dat)");
  if (st != PIKO_OK) {
    delete as;
    return st;
  }
  *out = as;
  return PIKO_OK;
}

piko_status piko_asset_info_get(const piko_asset* as, piko_asset_info* o)
{
  if (!as || !o) return PIKO_ERR_INVALID;
  memset(o, 0, sizeof(*o));
  const Asset& A = as->a;
  o->triangles = (int)A.tris.size();
  o->patches = (int)(A.patches.size() / 64);
  o->has_uv = A.has_uv ? 1 : 0;
  o->has_camera = A.cam.set ? 1 : 0;
  o->eye[0] = (float)A.cam.eye.x; o->eye[1] = (float)A.cam.eye.y; o->eye[2] = (float)A.cam.eye.z;
  o->target[0] = (float)A.cam.target.x; o->target[1] = (float)A.cam.target.y; o->target[2] = (float)A.cam.target.z;
  o->up[0] = (float)A.cam.up.x; o->up[1] = (float)A.cam.up.y; o->up[2] = (float)A.cam.up.z;
  o->fovy_rad = (float)A.cam.fovy;
  o->znear = (float)A.cam.znear;
  o->zfar = (float)A.cam.zfar;
  o->lights = (int)A.lights.size();
  if (!A.lights.empty()) memcpy(o->light_pos, A.lights[0].data(), sizeof(o->light_pos));
  o->materials = (int)A.diffuse.size();
  return PIKO_OK;
}

piko_status piko_asset_triangles(const piko_asset* as, int colour_source, float* pos, float* nrm, float* col, float* uv)
{
  if (!as || (colour_source != 0 && colour_source != 1)) return PIKO_ERR_INVALID;
  const std::vector<Tri>& T = as->a.tris;
  const size_t N = T.size();
  for (size_t t = 0; t < N; ++t)
    for (int k = 0; k < 3; ++k) {
      const size_t i = (size_t)k * N + t;
      if (pos) { for (int r = 0; r < 3; ++r) pos[4 * i + r] = T[t].p[k][r]; pos[4 * i + 3] = 1.0f; }
      if (nrm) { for (int r = 0; r < 3; ++r) nrm[4 * i + r] = T[t].n[k][r]; nrm[4 * i + 3] = 0.0f; }
      if (col) {
        // 0: the reference's fixed material colour (main.cpp:383), 1: the scene's material
        const float ref[3] = {0.9f, 0.9f, 0.6f};
        for (int r = 0; r < 3; ++r) col[4 * i + r] = colour_source ? T[t].col[r] : ref[r];
        col[4 * i + 3] = 1.0f;
      }
      if (uv) { uv[2 * i] = T[t].t[k][0]; uv[2 * i + 1] = T[t].t[k][1]; }
    }
  return PIKO_OK;
}

piko_status piko_asset_patches(const piko_asset* as, float* patches)
{
  if (!as || !patches) return PIKO_ERR_INVALID;
  memcpy(patches, as->a.patches.data(), as->a.patches.size() * sizeof(float));
  return PIKO_OK;
}

piko_status piko_asset_view_proj(const piko_asset* as, int width, int height, float* out16)
{
  if (!as || !out16 || width <= 0 || height <= 0) return PIKO_ERR_INVALID;
  view_proj(as->a.cam, width, height, out16);
  return PIKO_OK;
}

// 24-bit BMP of an RGBA8 image (R in the low byte, row 0 = bottom, as
// PikoScreen stores it; the reference writes screenshots with EasyBMP).  BMP
// rows are stored bottom-up, so image row 0 is the file's first row.
piko_status piko_image_write_bmp(const char* path, const uint32_t* rgba, int width, int height)
{
  if (!path || !rgba || width <= 0 || height <= 0 || width > 65536 || height > 65536) return fail("bad image");
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(std::string("cannot write ") + path);
  const uint32_t row = ((uint32_t)width * 3u + 3u) & ~3u;
  const uint32_t data = row * (uint32_t)height, size = 54u + data;
  unsigned char h[54] = {'B', 'M'};
  auto put32 = [&](int at, uint32_t v) { for (int k = 0; k < 4; ++k) h[at + k] = (unsigned char)(v >> (8 * k)); };
  put32(2, size);
  put32(10, 54);
  put32(14, 40);
  put32(18, (uint32_t)width);
  put32(22, (uint32_t)height);
  h[26] = 1;   // planes
  h[28] = 24;  // bits per pixel
  put32(34, data);
  put32(38, 2835);
  put32(42, 2835);
  bool ok = std::fwrite(h, 1, 54, f) == 54;
  std::vector<unsigned char> line(row, 0);
  for (int y = 0; y < height && ok; ++y) {
    for (int x = 0; x < width; ++x) {
      const uint32_t c = rgba[(size_t)y * width + x];
      line[3 * x + 0] = (unsigned char)(c >> 16);  // B
      line[3 * x + 1] = (unsigned char)(c >> 8);   // G
      line[3 * x + 2] = (unsigned char)c;          // R
    }
    ok = std::fwrite(line.data(), 1, row, f) == row;
  }
  if (std::fclose(f) != 0) ok = false;
  return ok ? PIKO_OK : fail(std::string("write failed: ") + path);
}

piko_status piko_asset_destroy(piko_asset* as)
{
  if (!as) return PIKO_ERR_INVALID;
  delete as;
  return PIKO_OK;
}

}  // extern "C"
