// Network-config JSON parsing and .npy reading for libnwprt.
//
// The reference parses config_comp.json with nlohmann::json (tinycudann/tcnn.cu:53-56)
// and reads weights with npy.h (Renderer/npy.h).  Neither is needed here: this is a
// small strict JSON reader for the five keys the relight network uses
// (vtx_enc / cmp_enc / out_prd / cmp_net / wve_enc, prt_network.h:39-42) and a
// little-endian .npy reader for C-ordered float32 / int32 arrays.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>

#include "nwprt_internal.cuh"

namespace nwprt {
namespace {

struct JVal {
  enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
  bool b = false;
  double num = 0;
  std::string str;
  std::vector<JVal> arr;
  std::map<std::string, JVal> obj;
};

struct JParser {
  const std::string& s;
  size_t i = 0;
  explicit JParser(const std::string& t) : s(t) {}

  [[noreturn]] void bad(const char* what) {
    fail(NWPRT_INVALID_ARG, std::string("config JSON: ") + what + " at offset " + std::to_string(i));
  }
  void ws() {
    while (i < s.size() && (s[i] == ' ' || s[i] == '\n' || s[i] == '\r' || s[i] == '\t')) ++i;
  }
  bool lit(const char* w) {
    size_t n = strlen(w);
    if (s.compare(i, n, w) == 0) { i += n; return true; }
    return false;
  }
  JVal value(int depth) {
    if (depth > 32) bad("nesting too deep");
    ws();
    if (i >= s.size()) bad("unexpected end");
    JVal v;
    char c = s[i];
    if (c == '{') {
      v.kind = JVal::Obj;
      ++i;
      ws();
      if (i < s.size() && s[i] == '}') { ++i; return v; }
      for (;;) {
        ws();
        if (i >= s.size() || s[i] != '"') bad("expected key");
        std::string k = string();
        ws();
        if (i >= s.size() || s[i] != ':') bad("expected ':'");
        ++i;
        v.obj[k] = value(depth + 1);
        ws();
        if (i < s.size() && s[i] == ',') { ++i; continue; }
        if (i < s.size() && s[i] == '}') { ++i; return v; }
        bad("expected ',' or '}'");
      }
    }
    if (c == '[') {
      v.kind = JVal::Arr;
      ++i;
      ws();
      if (i < s.size() && s[i] == ']') { ++i; return v; }
      for (;;) {
        v.arr.push_back(value(depth + 1));
        ws();
        if (i < s.size() && s[i] == ',') { ++i; continue; }
        if (i < s.size() && s[i] == ']') { ++i; return v; }
        bad("expected ',' or ']'");
      }
    }
    if (c == '"') { v.kind = JVal::Str; v.str = string(); return v; }
    if (lit("true")) { v.kind = JVal::Bool; v.b = true; return v; }
    if (lit("false")) { v.kind = JVal::Bool; v.b = false; return v; }
    if (lit("null")) return v;
    const char* b = s.c_str() + i;
    char* e = nullptr;
    double d = strtod(b, &e);
    if (e == b) bad("invalid value");
    i += (size_t)(e - b);
    v.kind = JVal::Num;
    v.num = d;
    return v;
  }
  std::string string() {
    std::string out;
    ++i;  // opening quote
    while (i < s.size() && s[i] != '"') {
      if (s[i] == '\\') {
        ++i;
        if (i >= s.size()) bad("bad escape");
        char e = s[i];
        out.push_back(e == 'n' ? '\n' : e == 't' ? '\t' : e);
      } else {
        out.push_back(s[i]);
      }
      ++i;
    }
    if (i >= s.size()) bad("unterminated string");
    ++i;
    return out;
  }
};

const JVal* get(const JVal& o, const char* k) {
  if (o.kind != JVal::Obj) return nullptr;
  auto it = o.obj.find(k);
  return it == o.obj.end() ? nullptr : &it->second;
}

double num(const JVal& o, const char* k, double dflt) {
  const JVal* v = get(o, k);
  if (!v) return dflt;
  if (v->kind != JVal::Num) fail(NWPRT_INVALID_ARG, std::string("config key '") + k + "' must be a number");
  return v->num;
}

int inum(const JVal& o, const char* k, int dflt) {
  double d = num(o, k, dflt);
  if (d != std::floor(d) || std::fabs(d) > 1e9)
    fail(NWPRT_INVALID_ARG, std::string("config key '") + k + "' must be an integer");
  return (int)d;
}

std::string str(const JVal& o, const char* k, const char* dflt) {
  const JVal* v = get(o, k);
  if (!v) return dflt;
  if (v->kind != JVal::Str) fail(NWPRT_INVALID_ARG, std::string("config key '") + k + "' must be a string");
  return v->str;
}

void mlp_shapes(int n_in, int width, int n_hidden, int n_out, int* nl, int* in, int* out) {
  if (n_hidden == 0) {
    *nl = 1;
    in[0] = n_in;
    out[0] = n_out;
    return;
  }
  if (n_hidden + 1 > kMaxLayers) fail(NWPRT_UNSUPPORTED, "too many hidden layers");
  *nl = n_hidden + 1;
  in[0] = n_in;
  out[0] = width;
  for (int l = 1; l < n_hidden; ++l) { in[l] = width; out[l] = width; }
  in[n_hidden] = width;
  out[n_hidden] = n_out;
}

}  // namespace

double NetDims::flops_per_eval() const {
  double f = 0;
  for (int i = 0; i < op_nl; ++i) f += 2.0 * op_in[i] * op_outs[i];
  for (int i = 0; i < cn_nl; ++i) f += 2.0 * (i == 0 ? op_out : cn_in[i]) * cn_outs[i];
  return f;
}

NetDims parse_config(const std::string& text) {
  JParser p(text);
  JVal root = p.value(0);
  p.ws();
  if (p.i != text.size()) p.bad("trailing characters");
  if (root.kind != JVal::Obj) fail(NWPRT_INVALID_ARG, "config JSON must be an object");
  static const JVal empty_obj = [] { JVal v; v.kind = JVal::Obj; return v; }();
  const JVal* ve = get(root, "vtx_enc");
  const JVal* op = get(root, "out_prd");
  const JVal* cn = get(root, "cmp_net");
  if (!ve || !op || !cn) fail(NWPRT_INVALID_ARG, "config needs vtx_enc, out_prd and cmp_net");
  const JVal* ce = get(root, "cmp_enc");
  const JVal* we = get(root, "wve_enc");
  if (!ce) ce = &empty_obj;
  if (!we) we = &empty_obj;
  if (str(*ve, "otype", "HashGrid") != "HashGrid") fail(NWPRT_UNSUPPORTED, "vtx_enc.otype must be HashGrid");
  if (str(*ce, "otype", "Identity") != "Identity") fail(NWPRT_UNSUPPORTED, "cmp_enc.otype must be Identity");
  for (const JVal* n : {op, cn}) {
    if (str(*n, "activation", "ReLU") != "ReLU") fail(NWPRT_UNSUPPORTED, "MLP activation must be ReLU");
    if (str(*n, "output_activation", "None") != "None")
      fail(NWPRT_UNSUPPORTED, "MLP output_activation must be None");
  }
  NetDims d;
  d.n_levels = inum(*ve, "n_levels", 16);
  d.n_features = inum(*ve, "n_features_per_level", 2);
  d.log2_table = inum(*ve, "log2_hashmap_size", 19);
  d.base_resolution = inum(*ve, "base_resolution", 16);
  d.per_level_scale = num(*ve, "per_level_scale", 2.0);
  d.aux_width = inum(*ce, "n_padded_dims", 16);
  d.op_neurons = inum(*op, "n_neurons", 64);
  d.op_hidden = inum(*op, "n_hidden_layers", 2);
  d.op_out = inum(*op, "n_output_dims", 64);
  d.cn_neurons = inum(*cn, "n_neurons", 64);
  d.cn_hidden = inum(*cn, "n_hidden_layers", 2);
  d.face_size = inum(*we, "face_size", 64);
  if (d.n_levels < 1 || d.n_levels > kMaxLevels) fail(NWPRT_INVALID_ARG, "n_levels out of range");
  if (d.n_features < 1 || d.n_features > 8) fail(NWPRT_INVALID_ARG, "n_features_per_level out of range");
  if (d.log2_table < 1 || d.log2_table > 24) fail(NWPRT_INVALID_ARG, "log2_hashmap_size out of range");
  if (d.base_resolution < 1 || !(d.per_level_scale >= 1.0))
    fail(NWPRT_INVALID_ARG, "base_resolution / per_level_scale out of range");
  if (d.aux_width < 13 || d.aux_width > 64) fail(NWPRT_INVALID_ARG, "cmp_enc.n_padded_dims must be in [13, 64]");
  if (d.face_size < 1 || d.face_size > 1024 || (d.face_size & (d.face_size - 1)))
    fail(NWPRT_INVALID_ARG, "wve_enc.face_size must be a power of two <= 1024");
  if (d.op_neurons < 1 || d.op_neurons > 256 || d.cn_neurons < 1 || d.cn_neurons > 256 ||
      d.op_out < 1 || d.op_out > 256 || d.op_hidden < 0 || d.cn_hidden < 0)
    fail(NWPRT_INVALID_ARG, "MLP dimensions out of range");
  const uint64_t T = 1ull << d.log2_table;
  uint64_t off = 0;
  for (int l = 0; l < d.n_levels; ++l) {
    double s = std::floor((double)d.base_resolution * std::pow(d.per_level_scale, (double)l));
    if (s < 1 || s > 1e6) fail(NWPRT_INVALID_ARG, "hash grid level resolution out of range");
    int n = (int)s;
    uint64_t v = (uint64_t)(n + 1) * (n + 1) * (n + 1);
    d.level_res[l] = n;
    d.level_size[l] = (int)(v < T ? v : T);
    d.level_offset[l] = (int)off;
    off += (uint64_t)d.level_size[l];
  }
  if (off * d.n_features > (1ull << 31)) fail(NWPRT_INVALID_ARG, "hash grid too large");
  mlp_shapes(d.enc_dims(), d.op_neurons, d.op_hidden, d.op_out, &d.op_nl, d.op_in, d.op_outs);
  mlp_shapes(d.op_out + d.aux_width, d.cn_neurons, d.cn_hidden, 3, &d.cn_nl, d.cn_in, d.cn_outs);
  return d;
}

NpyArray read_npy(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) fail(NWPRT_IO_ERROR, "cannot open " + path);
  char magic[8];
  f.read(magic, 8);
  if (!f || memcmp(magic, "\x93NUMPY", 6) != 0) fail(NWPRT_IO_ERROR, path + ": not a .npy file");
  uint32_t hlen = 0;
  if (magic[6] == 1) {
    unsigned char b[2];
    f.read((char*)b, 2);
    hlen = b[0] | (b[1] << 8);
  } else {
    unsigned char b[4];
    f.read((char*)b, 4);
    hlen = b[0] | (b[1] << 8) | (b[2] << 16) | ((uint32_t)b[3] << 24);
  }
  if (!f || hlen > (1u << 20)) fail(NWPRT_IO_ERROR, path + ": bad header");
  std::string h(hlen, '\0');
  f.read(&h[0], hlen);
  NpyArray a;
  auto field = [&](const char* key) -> std::string {
    size_t p = h.find(key);
    if (p == std::string::npos) fail(NWPRT_IO_ERROR, path + ": header lacks " + key);
    p = h.find(':', p);
    return h.substr(p + 1);
  };
  std::string d = field("'descr'");
  size_t q0 = d.find('\''), q1 = d.find('\'', q0 + 1);
  a.descr = d.substr(q0 + 1, q1 - q0 - 1);
  std::string fo = field("'fortran_order'");
  if (fo.find("True") < fo.find(',')) fail(NWPRT_IO_ERROR, path + ": fortran order unsupported");
  std::string sh = field("'shape'");
  size_t l = sh.find('('), r = sh.find(')');
  std::stringstream ss(sh.substr(l + 1, r - l - 1));
  std::string tok;
  size_t count = 1;
  while (std::getline(ss, tok, ',')) {
    if (tok.find_first_not_of(" ") == std::string::npos) continue;
    size_t v = std::stoull(tok);
    a.shape.push_back(v);
    count *= v;
  }
  size_t elem = 0;
  if (a.descr == "<f4" || a.descr == "<i4") elem = 4;
  else fail(NWPRT_IO_ERROR, path + ": dtype " + a.descr + " unsupported (need <f4 or <i4)");
  a.data.resize(count * elem);
  f.read(a.data.data(), (std::streamsize)a.data.size());
  if (!f) fail(NWPRT_IO_ERROR, path + ": truncated data");
  return a;
}

}  // namespace nwprt
