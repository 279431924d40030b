// jlser.cpp -- the reference's index file: a Julia `Serialization` stream of
// one NamedTuple.  The reference writes it with `serialize(io, nt)`
// (RotorMap/common/dna.jl:23-34 `save` / `load`) for the NamedTuple that
// _index_data_nt builds (RotorMap/index/build.jl:755-772):
//   fp8 layout  ("indexreal.fp8.v1"): format, source, k, kstep, s, m, c,
//               normalize, fp8, n_frag, embeds8::Matrix{Float8_E4M3FN}
//               (rdim, N), norms::Matrix{Float32} (m, N), heads::Vector{String},
//               starts::Vector{Int}, strand::Vector{UInt8};
//   row layout  ("indexreal.v1"): the same with fp16::Bool and
//               embeds::Matrix{Float16 or Float32} (N, rdim).
//
// The stream format is the one of Julia's Serialization standard library
// (Julia 1.12.2 is the reference's toolchain, RotorMap/Manifest.toml:3).
// Only the subset such a NamedTuple uses is read and written here:
//   * an 8-byte header: HEADER tag, "JL", format version, flags (bit 0-1
//     endianness, bits 2-3 word size), three reserved bytes;
//   * one byte per tag; a tag is the 1-based position of a type or value in
//     the library's fixed TAGS table.  Tags >= VALUE_TAGS (the position of
//     `()`) are values by themselves: (), Bool, false, true, nothing, a fixed
//     list of common symbols, and the Int32 / Int64 literals 0..32.  A type
//     whose tag is below VALUE_TAGS, written as a value, is a 0 byte and then
//     its tag;
//   * symbols (SYMBOL + u8 length, LONGSYMBOL + i32 length), strings (STRING
//     + u8 length, LONGSTRING + i32 length), Int64 (a literal, SHORTINT64 +
//     i32, or INT64 + 8 bytes), tuples (TUPLE + u8 count, LONGTUPLE + i32);
//   * a module: MODULE, the root package's UUID as a UInt128 (or nothing for
//     Core / Main), its name, submodule names, then ();
//   * a DataType: DATATYPE, its name, its module and, for a parametric type,
//     an i32 parameter count and the parameters;
//   * an immutable struct (the NamedTuple): OBJECT, its type, its fields;
//   * an Array: ARRAY, the element type (omitted for UInt8), the length
//     (vectors) or the dims tuple, then the raw column-major elements for a
//     bits type or one object per element otherwise;
//   * back-references: every DataType, Array, Symbol longer than 7 bytes and
//     String longer than 7 bytes takes the next id of a counter when first
//     written (a String through a SHARED_REF tag); a later occurrence of the
//     same object is SHORTBACKREF + u16 id (BACKREF + i32, LONGBACKREF + i64
//     for larger ids).  The heads vector repeats its record header for every
//     window, so all but the first occurrence of each header are back-
//     references.
// Bulk arrays are returned as pointers into the memory-mapped file, so a
// 6 GiB embeds8 costs no copy before its single host-to-device transfer.
#include <fcntl.h>
#include <stdio.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "r2m.h"

namespace r2m {
int fail(int code, const std::string &msg);
}  // namespace r2m

namespace {

// Positions in Julia's Serialization TAGS table (1-based, as written).
enum : uint8_t {
  T_SYMBOL = 1, T_INT8 = 2, T_UINT8 = 3, T_INT16 = 4, T_UINT16 = 5, T_INT32 = 6, T_UINT32 = 7,
  T_INT64 = 8, T_UINT64 = 9, T_INT128 = 10, T_UINT128 = 11, T_FLOAT16 = 12, T_FLOAT32 = 13,
  T_FLOAT64 = 14, T_CHAR = 15, T_DATATYPE = 16, T_TUPLE = 20, T_ARRAY = 21, T_MODULE = 31,
  T_STRING = 33,
  T_UNDEFREF = 41, T_BACKREF = 42, T_LONGBACKREF = 43, T_SHORTBACKREF = 44, T_LONGTUPLE = 45,
  T_LONGSYMBOL = 46, T_LONGSTRING = 48, T_SHORTINT64 = 49, T_FULL_DATATYPE = 50,
  T_WRAPPER_DATATYPE = 51, T_OBJECT = 52, T_REF_OBJECT = 53, T_HEADER = 55, T_SHARED_REF = 57,
  // values that are their own tag
  T_EMPTYTUPLE = 68, T_BOOL_TYPE = 69, T_ANY_TYPE = 70, T_FALSE = 76, T_TRUE = 77, T_NOTHING = 78,
  T_SYM0 = 79,        // first of the fixed symbols
  T_RESERVED0 = 166,  // 24 reserved slots
  T_ZERO32 = 190,     // Int32 literals 0..32
  T_ZERO64 = 223,     // Int64 literals 0..32
};
constexpr int kIntLiterals = 33;
// Format version written by r2m_jlbin_write.  Julia refuses a stream whose
// version is newer than its own and reads older ones; none of the tags an
// index file uses changed encoding in later versions.
constexpr uint8_t kWriteVersion = 20;

// The fixed symbols of the TAGS table, tags 79..165, in table order.
const char *const kSyms[] = {
    "Any", "Array", "TypeVar", "Box", "Tuple", "Ptr", "return", "call", "::", "Function", "=", "==", "===",
    "gotoifnot", "A", "B", "C", "M", "N", "T", "S", "X", "Y", "a", "b", "c", "d", "e", "f", "g", "h", "i", "j",
    "k", "l", "m", "n", "o", "p", "q", "r", "s", "t", "u", "v", "w", "x", "y", "z", "add_int", "sub_int",
    "mul_int", "add_float", "sub_float", "new", "mul_float", "bitcast", "start", "done", "next",
    "indexed_iterate", "getfield", "meta", "eq_int", "slt_int", "sle_int", "ne_int", "push_loc", "pop_loc",
    "pop", "arrayset", "arrayref", "apply_type", "inbounds", "getindex", "setindex!", "Core", "!", "+", "Base",
    "static_parameter", "convert", "colon", "#self#", "#temp#", "tuple", ""};
constexpr int kNSyms = (int)(sizeof(kSyms) / sizeof(kSyms[0]));
static_assert(kNSyms == T_RESERVED0 - T_SYM0, "symbol table must fill tags 79..165");

int sym_tag(const std::string &s) {
  for (int i = 0; i < kNSyms; ++i)
    if (s == kSyms[i]) return T_SYM0 + i;
  return 0;
}

// The DLFP8Types package (RotorMap/Manifest.toml:339-342) that defines
// Float8_E4M3FN, the element type of embeds8.
const char *const kFp8Pkg = "DLFP8Types";
const char *const kFp8PkgUuid = "f4c16678-4a16-415b-82ef-ed337c5d6c7c";

// ------------------------------------------------------------ object model

struct JObj;
using JP = std::shared_ptr<JObj>;

struct JObj {
  enum Kind { NOTHING, EMPTYTUPLE, BOOL, INT, UINT128, FLOAT, SYM, STR, TYPE, MODULE, TUPLE, ARRAY, NTUPLE };
  Kind kind;
  explicit JObj(Kind k) : kind(k) {}
  int64_t i = 0;           // INT, BOOL
  uint64_t lo = 0, hi = 0;  // UINT128
  double f = 0;            // FLOAT
  std::string s;           // SYM, STR; TYPE name; MODULE root name
  int builtin = 0;         // TYPE: its TAGS position when it has one (String, Int64, ...)
  std::vector<std::string> modpath;  // TYPE: module path; MODULE: path
  std::vector<JP> items;   // TUPLE items; TYPE parameters; NTUPLE values
  std::vector<std::string> names;    // NTUPLE field names
  // ARRAY
  JP elty;
  std::vector<int64_t> dims;
  const uint8_t *data = nullptr;
  size_t nbytes = 0;
  std::vector<int32_t> sidx;      // string arrays: per element, index into uniq
  std::vector<std::string> uniq;  // string arrays: distinct strings, first-seen order
  // string objects met inside a string array: the array they were indexed for
  const JObj *owner = nullptr;
  int32_t uidx = -1;
};

JP mk(JObj::Kind k) { return std::make_shared<JObj>(k); }

int elem_size(const JObj &t) {
  if (t.kind != JObj::TYPE) return 0;
  switch (t.builtin) {
    case T_INT8: case T_UINT8: return 1;
    case T_INT16: case T_UINT16: case T_FLOAT16: return 2;
    case T_INT32: case T_UINT32: case T_FLOAT32: case T_CHAR: return 4;
    case T_INT64: case T_UINT64: case T_FLOAT64: return 8;
    case T_INT128: case T_UINT128: return 16;
    default: break;
  }
  if (t.builtin == 0 && t.s == "Float8_E4M3FN") return 1;
  return 0;
}

// Names of parametric types an index file may contain (their DATATYPE entry
// carries a parameter count); every other named type must be a known
// non-parametric one.
bool is_parametric(const std::string &name) {
  return name == "NamedTuple" || name == "Tuple" || name == "Array";
}
bool is_known_plain(const std::string &name) { return name == "Float8_E4M3FN"; }

// ------------------------------------------------------------------ reader

struct ParseError {
  std::string msg;
};

struct Reader {
  const uint8_t *base, *p, *end;
  std::vector<JP> table;
  int64_t counter = 0;
  int version = -1;

  void need(size_t n) {
    if ((size_t)(end - p) < n) throw ParseError{"unexpected end of stream at byte " + std::to_string(p - base)};
  }
  uint8_t u8() { need(1); return *p++; }
  template <typename T>
  T raw() {
    need(sizeof(T));
    T v;
    memcpy(&v, p, sizeof(T));
    p += sizeof(T);
    return v;
  }
  int64_t slot() { return counter++; }
  void set(int64_t id, JP o) {
    if ((int64_t)table.size() <= id) table.resize(id + 1);
    table[id] = std::move(o);
  }
  JP ref(int64_t id) {
    if (id < 0 || id >= (int64_t)table.size() || !table[id])
      throw ParseError{"back-reference to unknown id " + std::to_string(id)};
    return table[id];
  }

  JP obj() { return handle(u8()); }

  JP sym(size_t len) {
    need(len);
    JP o = mk(JObj::SYM);
    o->s.assign(reinterpret_cast<const char *>(p), len);
    p += len;
    if (len > 7) set(slot(), o);
    return o;
  }
  JP str(size_t len) {
    need(len);
    JP o = mk(JObj::STR);
    o->s.assign(reinterpret_cast<const char *>(p), len);
    p += len;
    return o;
  }
  JP type_builtin(int tag) {
    JP o = mk(JObj::TYPE);
    o->builtin = tag;
    return o;
  }
  JP intv(int64_t v) {
    JP o = mk(JObj::INT);
    o->i = v;
    return o;
  }

  JP handle(uint8_t b) {
    if (b == 0) {  // a type (or other TAGS entry) written as a value
      uint8_t t = u8();
      if (t == 0 || t >= T_EMPTYTUPLE) throw ParseError{"bad escaped tag " + std::to_string(t)};
      return type_builtin(t);
    }
    if (b >= T_EMPTYTUPLE) return value_tag(b);
    switch (b) {
      case T_TUPLE: return tuple(u8());
      case T_LONGTUPLE: return tuple((size_t)raw<int32_t>());
      case T_SHORTBACKREF: return ref(raw<uint16_t>());
      case T_BACKREF: return ref(raw<int32_t>());
      case T_LONGBACKREF: return ref(raw<int64_t>());
      case T_ARRAY: return array();
      case T_DATATYPE: return datatype();
      case T_OBJECT: return object(obj());
      case T_SHARED_REF: {
        int64_t id = slot();
        JP o = obj();
        set(id, o);
        return o;
      }
      case T_SYMBOL: return sym(u8());
      case T_LONGSYMBOL: return sym((size_t)raw<int32_t>());
      case T_SHORTINT64: return intv(raw<int32_t>());
      case T_MODULE: return module();
      case T_STRING: return str(u8());
      case T_LONGSTRING: return str((size_t)raw<int32_t>());
      case T_HEADER: header(); return obj();
      case T_INT8: return intv(raw<int8_t>());
      case T_UINT8: return intv(raw<uint8_t>());
      case T_INT16: return intv(raw<int16_t>());
      case T_UINT16: return intv(raw<uint16_t>());
      case T_INT32: return intv(raw<int32_t>());
      case T_UINT32: return intv(raw<uint32_t>());
      case T_INT64: return intv(raw<int64_t>());
      case T_UINT64: {
        uint64_t v = raw<uint64_t>();
        if (v > (uint64_t)INT64_MAX) throw ParseError{"UInt64 value out of Int64 range"};
        return intv((int64_t)v);
      }
      case T_UINT128: case T_INT128: {
        JP o = mk(JObj::UINT128);
        o->lo = raw<uint64_t>();
        o->hi = raw<uint64_t>();
        return o;
      }
      case T_FLOAT32: { JP o = mk(JObj::FLOAT); o->f = raw<float>(); return o; }
      case T_FLOAT64: { JP o = mk(JObj::FLOAT); o->f = raw<double>(); return o; }
      case T_FULL_DATATYPE: case T_WRAPPER_DATATYPE:
        throw ParseError{"whole-type serialization (anonymous functions) is not part of an index file"};
      case T_REF_OBJECT:
        throw ParseError{"mutable objects are not part of an index file"};
      default:
        throw ParseError{"unsupported tag " + std::to_string(b) + " at byte " + std::to_string(p - base - 1)};
    }
  }

  JP value_tag(uint8_t b) {
    if (b == T_EMPTYTUPLE) return mk(JObj::EMPTYTUPLE);
    if (b == T_BOOL_TYPE || b == T_ANY_TYPE) return type_builtin(b);
    if (b == T_FALSE || b == T_TRUE) {
      JP o = mk(JObj::BOOL);
      o->i = b == T_TRUE;
      return o;
    }
    if (b == T_NOTHING) return mk(JObj::NOTHING);
    if (b >= T_SYM0 && b < T_RESERVED0) {
      JP o = mk(JObj::SYM);
      o->s = kSyms[b - T_SYM0];
      return o;
    }
    if (b >= T_ZERO32 && b < T_ZERO32 + kIntLiterals) return intv(b - T_ZERO32);
    if (b >= T_ZERO64) return intv(b - T_ZERO64);
    throw ParseError{"unsupported value tag " + std::to_string(b)};
  }

  void header() {
    uint8_t j = u8(), l = u8();
    if (j != 'J' || l != 'L') throw ParseError{"not a Julia serialization stream (bad magic)"};
    version = u8();
    uint8_t flags = u8();
    need(3);
    p += 3;
    if ((flags & 3) != 0) throw ParseError{"big-endian Julia streams are not supported"};
    if (((flags >> 2) & 3) != 1) throw ParseError{"only 64-bit Julia streams are supported"};
  }

  JP tuple(size_t n) {
    JP o = mk(JObj::TUPLE);
    need(n);  // every element takes at least one byte
    o->items.reserve(n);
    for (size_t i = 0; i < n; ++i) o->items.push_back(obj());
    return o;
  }

  JP module() {
    JP o = mk(JObj::MODULE);
    JP key = obj();
    if (key->kind == JObj::TUPLE) {  // the oldest format: a tuple of names
      for (auto &it : key->items) {
        if (it->kind != JObj::SYM) throw ParseError{"bad module path"};
        o->modpath.push_back(it->s);
      }
      if (o->modpath.empty()) o->modpath.push_back("Main");
      return o;
    }
    if (key->kind != JObj::NOTHING && key->kind != JObj::UINT128) throw ParseError{"bad module key"};
    JP name = obj();
    if (name->kind != JObj::SYM) throw ParseError{"bad module name"};
    o->modpath.push_back(name->s);
    for (;;) {
      JP sub = obj();
      if (sub->kind == JObj::EMPTYTUPLE) break;
      if (sub->kind != JObj::SYM) throw ParseError{"bad submodule name"};
      o->modpath.push_back(sub->s);
    }
    return o;
  }

  JP datatype() {
    int64_t id = slot();
    JP a = obj(), b = obj();
    JP name = a->kind == JObj::SYM ? a : b, mod = a->kind == JObj::SYM ? b : a;
    if (name->kind != JObj::SYM || mod->kind != JObj::MODULE) throw ParseError{"bad DataType entry"};
    JP t = mk(JObj::TYPE);
    t->s = name->s;
    t->modpath = mod->modpath;
    if (is_parametric(t->s)) {
      int32_t np = raw<int32_t>();
      if (np < 0 || np > 4096) throw ParseError{"bad parameter count"};
      for (int32_t i = 0; i < np; ++i) t->items.push_back(obj());
    } else if (!is_known_plain(t->s)) {
      throw ParseError{"type " + t->s + " is not part of an index file"};
    }
    set(id, t);
    return t;
  }

  JP array() {
    int64_t id = slot();
    JP arr = mk(JObj::ARRAY);
    set(id, arr);
    JP d1 = obj();
    if (d1->kind == JObj::TYPE) {
      arr->elty = d1;
      d1 = obj();
    } else {
      arr->elty = type_builtin(T_UINT8);
    }
    if (d1->kind == JObj::INT) {
      arr->dims.push_back(d1->i);
    } else if (d1->kind == JObj::TUPLE) {
      for (auto &it : d1->items) {
        if (it->kind != JObj::INT) throw ParseError{"bad array dims"};
        arr->dims.push_back(it->i);
      }
    } else {
      throw ParseError{"bad array dims"};
    }
    size_t n = 1;
    for (int64_t d : arr->dims) {
      if (d < 0) throw ParseError{"negative array dimension"};
      if (__builtin_mul_overflow(n, (size_t)d, &n)) throw ParseError{"array dimensions overflow"};
    }
    const int es = elem_size(*arr->elty);
    if (es > 0) {
      if (__builtin_mul_overflow(n, (size_t)es, &arr->nbytes)) throw ParseError{"array size overflows"};
      need(arr->nbytes);
      arr->data = p;
      p += arr->nbytes;
      return arr;
    }
    if (!(arr->elty->kind == JObj::TYPE && arr->elty->builtin == T_STRING))
      throw ParseError{"array element type is not part of an index file"};
    string_elements(*arr, n);
    return arr;
  }

  // Vector{String} elements, the one hot loop (a column count of entries).
  void string_elements(JObj &arr, size_t n) {
    need(n);  // every element takes at least one byte
    arr.sidx.resize(n);
    std::unordered_map<std::string, int32_t> inline_ids;
    auto intern_obj = [&](JObj *s) -> int32_t {
      if (s->owner != &arr) {
        s->owner = &arr;
        s->uidx = (int32_t)arr.uniq.size();
        arr.uniq.push_back(s->s);
      }
      return s->uidx;
    };
    for (size_t e = 0; e < n; ++e) {
      uint8_t b = u8();
      if (b == T_STRING || b == T_LONGSTRING) {  // short strings: written in full each time
        size_t len = b == T_STRING ? u8() : (size_t)raw<int32_t>();
        need(len);
        std::string s(reinterpret_cast<const char *>(p), len);
        p += len;
        auto it = inline_ids.find(s);
        int32_t u;
        if (it == inline_ids.end()) {
          u = (int32_t)arr.uniq.size();
          arr.uniq.push_back(s);
          inline_ids.emplace(std::move(s), u);
        } else {
          u = it->second;
        }
        arr.sidx[e] = u;
        continue;
      }
      if (b == T_UNDEFREF) throw ParseError{"undefined string element"};
      JP o = handle(b);
      if (o->kind != JObj::STR) throw ParseError{"string array holds a non-string element"};
      arr.sidx[e] = intern_obj(o.get());
    }
  }

  JP object(JP t) {
    if (t->kind != JObj::TYPE || t->s != "NamedTuple" || t->items.size() != 2)
      throw ParseError{"the index file must hold one NamedTuple"};
    const JP &names = t->items[0], &types = t->items[1];
    if (names->kind != JObj::TUPLE || types->kind != JObj::TYPE || types->s != "Tuple" ||
        types->items.size() != names->items.size())
      throw ParseError{"malformed NamedTuple type"};
    JP o = mk(JObj::NTUPLE);
    for (auto &nm : names->items) {
      if (nm->kind != JObj::SYM) throw ParseError{"NamedTuple field name is not a Symbol"};
      o->names.push_back(nm->s);
    }
    for (size_t i = 0; i < o->names.size(); ++i) {
      uint8_t b = u8();
      if (b == T_UNDEFREF) throw ParseError{"undefined NamedTuple field"};
      o->items.push_back(handle(b));
    }
    return o;
  }
};

int elty_code(const JObj &t) {
  if (t.kind != JObj::TYPE) return 0;
  switch (t.builtin) {
    case T_UINT8: return R2M_JL_U8;
    case T_INT32: return R2M_JL_I32;
    case T_INT64: return R2M_JL_I64;
    case T_FLOAT16: return R2M_JL_F16;
    case T_FLOAT32: return R2M_JL_F32;
    case T_FLOAT64: return R2M_JL_F64;
    default: break;
  }
  if (t.builtin == 0 && t.s == "Float8_E4M3FN") return R2M_JL_E4M3;
  return 0;
}

}  // namespace

struct r2m_jlbin {
  void *map = nullptr;
  size_t map_len = 0;
  const uint8_t *base = nullptr;
  int version = -1;
  JP nt;
  // per-field flattened strings of string arrays
  std::vector<std::string> blobs;
  std::vector<std::vector<int64_t>> offs;
};

static int jlbin_parse(r2m_jlbin *h, const uint8_t *data, size_t len) {
  Reader r{data, data, data + len};
  try {
    if (len == 0 || data[0] != T_HEADER) throw ParseError{"not a Julia serialization stream (no header tag)"};
    JP o = r.obj();
    if (o->kind != JObj::NTUPLE) throw ParseError{"the stream does not hold a NamedTuple"};
    h->nt = o;
    h->version = r.version;
  } catch (const ParseError &e) {
    return r2m::fail(R2M_EIO, "index .bin: " + e.msg);
  } catch (const std::bad_alloc &) {
    return r2m::fail(R2M_ENOMEM, "index .bin: out of host memory");
  } catch (const std::exception &e) {
    return r2m::fail(R2M_EIO, std::string("index .bin: ") + e.what());
  }
  h->base = data;
  const size_t nf = h->nt->items.size();
  h->blobs.resize(nf);
  h->offs.resize(nf);
  for (size_t i = 0; i < nf; ++i) {
    const JObj &v = *h->nt->items[i];
    if (v.kind != JObj::ARRAY || v.uniq.empty() && v.sidx.empty()) continue;
    std::string &b = h->blobs[i];
    std::vector<int64_t> &o = h->offs[i];
    o.reserve(v.uniq.size() + 1);
    for (const auto &s : v.uniq) {
      o.push_back((int64_t)b.size());
      b += s;
    }
    o.push_back((int64_t)b.size());
  }
  return R2M_OK;
}

extern "C" int r2m_jlbin_parse(const void *data, size_t len, r2m_jlbin **out) {
  if (!out) return r2m::fail(R2M_EINVAL, "out is null");
  *out = nullptr;
  if (!data && len) return r2m::fail(R2M_EINVAL, "data is null");
  std::unique_ptr<r2m_jlbin> h(new (std::nothrow) r2m_jlbin());
  if (!h) return r2m::fail(R2M_ENOMEM, "out of host memory");
  int rc = jlbin_parse(h.get(), static_cast<const uint8_t *>(data), len);
  if (rc) return rc;
  *out = h.release();
  return R2M_OK;
}

extern "C" int r2m_jlbin_open(const char *path, r2m_jlbin **out) {
  if (!out || !path) return r2m::fail(R2M_EINVAL, "null argument");
  *out = nullptr;
  int fd = ::open(path, O_RDONLY);
  if (fd < 0) return r2m::fail(R2M_EIO, std::string("cannot open index file ") + path);
  struct stat st;
  if (fstat(fd, &st) != 0 || st.st_size <= 0) {
    ::close(fd);
    return r2m::fail(R2M_EIO, std::string("empty or unreadable index file ") + path);
  }
  void *m = mmap(nullptr, (size_t)st.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
  ::close(fd);
  if (m == MAP_FAILED) return r2m::fail(R2M_EIO, std::string("cannot map index file ") + path);
  std::unique_ptr<r2m_jlbin> h(new (std::nothrow) r2m_jlbin());
  if (!h) {
    munmap(m, (size_t)st.st_size);
    return r2m::fail(R2M_ENOMEM, "out of host memory");
  }
  h->map = m;
  h->map_len = (size_t)st.st_size;
  int rc = jlbin_parse(h.get(), static_cast<const uint8_t *>(m), (size_t)st.st_size);
  if (rc) {
    munmap(m, (size_t)st.st_size);
    return rc;
  }
  *out = h.release();
  return R2M_OK;
}

extern "C" void r2m_jlbin_close(r2m_jlbin *h) {
  if (!h) return;
  if (h->map) munmap(h->map, h->map_len);
  delete h;
}

extern "C" int r2m_jlbin_version(const r2m_jlbin *h) { return h ? h->version : -1; }

extern "C" int r2m_jlbin_nfields(const r2m_jlbin *h) { return h && h->nt ? (int)h->nt->items.size() : 0; }

extern "C" int r2m_jlbin_field(const r2m_jlbin *h, int i, r2m_jl_field *out) {
  if (!h || !out || !h->nt) return r2m::fail(R2M_EINVAL, "null argument");
  if (i < 0 || i >= (int)h->nt->items.size()) return r2m::fail(R2M_EINVAL, "field index out of range");
  memset(out, 0, sizeof(*out));
  out->name = h->nt->names[i].c_str();
  out->offset = -1;
  const JObj &v = *h->nt->items[i];
  switch (v.kind) {
    case JObj::INT: out->kind = R2M_JL_INT; out->ival = v.i; break;
    case JObj::BOOL: out->kind = R2M_JL_BOOL; out->ival = v.i; break;
    case JObj::STR:
      out->kind = R2M_JL_STRING;
      out->str = v.s.data();
      out->str_len = (int64_t)v.s.size();
      break;
    case JObj::ARRAY:
      if (v.dims.size() > 2) {
        out->kind = R2M_JL_OTHER;
        break;
      }
      out->ndims = (int)v.dims.size();
      for (size_t d = 0; d < v.dims.size(); ++d) out->dims[d] = v.dims[d];
      if (v.data) {
        out->kind = R2M_JL_ARRAY;
        out->elty = elty_code(*v.elty);
        out->data = v.data;
        out->offset = (int64_t)(v.data - h->base);
      } else {
        out->kind = R2M_JL_STRVEC;
        out->data = v.sidx.data();
        out->blob = h->blobs[i].data();
        out->uniq_off = h->offs[i].data();
        out->nuniq = (int64_t)v.uniq.size();
      }
      break;
    default: out->kind = R2M_JL_OTHER; break;
  }
  return R2M_OK;
}

// ------------------------------------------------------------------ writer

namespace {

struct Writer {
  FILE *f;
  bool ok = true;
  int64_t counter = 0;
  std::unordered_map<std::string, int64_t> types, syms, strs;

  void bytes(const void *p, size_t n) {
    if (ok && n && fwrite(p, 1, n, f) != n) ok = false;
  }
  void u8(uint8_t v) { bytes(&v, 1); }
  template <typename T>
  void raw(T v) { bytes(&v, sizeof(T)); }

  void backref(int64_t id) {
    if (id <= 0xFFFF) {
      u8(T_SHORTBACKREF);
      raw<uint16_t>((uint16_t)id);
    } else if (id <= INT32_MAX) {
      u8(T_BACKREF);
      raw<int32_t>((int32_t)id);
    } else {
      u8(T_LONGBACKREF);
      raw<int64_t>(id);
    }
  }
  void int64(int64_t v) {
    if (v >= 0 && v < kIntLiterals) {
      u8((uint8_t)(T_ZERO64 + v));
    } else if (v >= INT32_MIN && v <= INT32_MAX) {
      u8(T_SHORTINT64);
      raw<int32_t>((int32_t)v);
    } else {
      u8(T_INT64);
      raw<int64_t>(v);
    }
  }
  void symbol(const std::string &s) {
    if (int t = sym_tag(s)) {
      u8((uint8_t)t);
      return;
    }
    if (s.size() > 7) {
      auto it = syms.find(s);
      if (it != syms.end()) {
        backref(it->second);
        return;
      }
      syms.emplace(s, counter++);
    }
    if (s.size() <= 255) {
      u8(T_SYMBOL);
      u8((uint8_t)s.size());
    } else {
      u8(T_LONGSYMBOL);
      raw<int32_t>((int32_t)s.size());
    }
    bytes(s.data(), s.size());
  }
  void string(const char *p, size_t n) {
    if (n > 7) {
      std::string key(p, n);
      auto it = strs.find(key);
      if (it != strs.end()) {
        backref(it->second);
        return;
      }
      strs.emplace(std::move(key), counter++);
      u8(T_SHARED_REF);
    }
    if (n <= 255) {
      u8(T_STRING);
      u8((uint8_t)n);
    } else {
      u8(T_LONGSTRING);
      raw<int32_t>((int32_t)n);
    }
    bytes(p, n);
  }
  void module_core() {
    u8(T_MODULE);
    u8(T_NOTHING);
    symbol("Core");
    u8(T_EMPTYTUPLE);
  }
  void module_fp8() {
    u8(T_MODULE);
    // the package UUID as its UInt128 value, little-endian
    uint64_t v[2] = {0, 0};
    int nib = 0;
    for (const char *c = kFp8PkgUuid; *c; ++c) {
      int d;
      if (*c >= '0' && *c <= '9') d = *c - '0';
      else if (*c >= 'a' && *c <= 'f') d = *c - 'a' + 10;
      else continue;
      // nibble `nib` counted from the most significant end of 128 bits
      const int bit = 124 - 4 * nib++;
      v[bit >= 64] |= (uint64_t)d << (bit & 63);
    }
    u8(T_UINT128);
    raw<uint64_t>(v[0]);
    raw<uint64_t>(v[1]);
    symbol(kFp8Pkg);
    u8(T_EMPTYTUPLE);
  }
  // An element type of an Array field.
  void elty(int code) {
    switch (code) {
      case R2M_JL_U8: u8(0); u8(T_UINT8); return;
      case R2M_JL_I32: u8(0); u8(T_INT32); return;
      case R2M_JL_I64: u8(0); u8(T_INT64); return;
      case R2M_JL_F16: u8(0); u8(T_FLOAT16); return;
      case R2M_JL_F32: u8(0); u8(T_FLOAT32); return;
      case R2M_JL_F64: u8(0); u8(T_FLOAT64); return;
      case 100: u8(0); u8(T_STRING); return;  // String
      default: break;
    }
    // Float8_E4M3FN: a plain DataType of the DLFP8Types package
    const std::string key = "Float8_E4M3FN";
    auto it = types.find(key);
    if (it != types.end()) {
      backref(it->second);
      return;
    }
    types.emplace(key, counter++);
    u8(T_DATATYPE);
    symbol("Float8_E4M3FN");
    module_fp8();
  }
  // Array{elty, ndims} as a type.
  void array_type(int code, int ndims) {
    const std::string key = "Array{" + std::to_string(code) + "," + std::to_string(ndims) + "}";
    auto it = types.find(key);
    if (it != types.end()) {
      backref(it->second);
      return;
    }
    types.emplace(key, counter++);
    u8(T_DATATYPE);
    symbol("Array");
    module_core();
    raw<int32_t>(2);
    elty(code);
    int64(ndims);
  }
  void field_type(const r2m_jl_field &fl) {
    switch (fl.kind) {
      case R2M_JL_INT: u8(0); u8(T_INT64); return;
      case R2M_JL_BOOL: u8(T_BOOL_TYPE); return;
      case R2M_JL_STRING: u8(0); u8(T_STRING); return;
      case R2M_JL_ARRAY: array_type(fl.elty, fl.ndims); return;
      case R2M_JL_STRVEC: array_type(100, 1); return;
      default: ok = false; return;
    }
  }
};

int jl_elem_size(int code) {
  switch (code) {
    case R2M_JL_U8: case R2M_JL_E4M3: return 1;
    case R2M_JL_F16: return 2;
    case R2M_JL_I32: case R2M_JL_F32: return 4;
    case R2M_JL_I64: case R2M_JL_F64: return 8;
    default: return 0;
  }
}

}  // namespace

extern "C" int r2m_jlbin_write(const char *path, const r2m_jl_field *fields, int nfields) {
  if (!path || (!fields && nfields)) return r2m::fail(R2M_EINVAL, "null argument");
  if (nfields < 1 || nfields > 255) return r2m::fail(R2M_EINVAL, "a NamedTuple of 1..255 fields is written");
  for (int i = 0; i < nfields; ++i) {
    const r2m_jl_field &fl = fields[i];
    if (!fl.name || !*fl.name) return r2m::fail(R2M_EINVAL, "field " + std::to_string(i) + " has no name");
    switch (fl.kind) {
      case R2M_JL_INT: case R2M_JL_BOOL: break;
      case R2M_JL_STRING:
        if (fl.str_len < 0 || (fl.str_len && !fl.str) || fl.str_len > INT32_MAX)
          return r2m::fail(R2M_EINVAL, std::string("bad string field ") + fl.name);
        break;
      case R2M_JL_ARRAY:
        if (!jl_elem_size(fl.elty) || fl.ndims < 1 || fl.ndims > 2 || fl.dims[0] < 0 ||
            (fl.ndims == 2 && fl.dims[1] < 0))
          return r2m::fail(R2M_EINVAL, std::string("bad array field ") + fl.name);
        if (!fl.data && fl.dims[0] * (fl.ndims == 2 ? fl.dims[1] : 1) > 0)
          return r2m::fail(R2M_EINVAL, std::string("array field without data: ") + fl.name);
        break;
      case R2M_JL_STRVEC:
        if (fl.ndims != 1 || fl.dims[0] < 0 || fl.nuniq < 0 || (fl.dims[0] && (!fl.data || !fl.uniq_off)) ||
            (fl.nuniq && (!fl.uniq_off || (fl.uniq_off[fl.nuniq] > 0 && !fl.blob))))
          return r2m::fail(R2M_EINVAL, std::string("bad string-vector field ") + fl.name);
        break;
      default: return r2m::fail(R2M_EINVAL, std::string("unsupported field kind for ") + fl.name);
    }
  }
  FILE *f = fopen(path, "wb");
  if (!f) return r2m::fail(R2M_EIO, std::string("cannot create ") + path);
  std::vector<char> buf(1 << 22);
  setvbuf(f, buf.data(), _IOFBF, buf.size());
  Writer w{f};
  // header
  const uint8_t hdr[8] = {T_HEADER, 'J', 'L', kWriteVersion, 1u << 2, 0, 0, 0};
  w.bytes(hdr, 8);
  // the NamedTuple's type
  w.u8(T_OBJECT);
  w.counter++;  // the NamedTuple{...} DataType
  w.u8(T_DATATYPE);
  w.symbol("NamedTuple");
  w.module_core();
  w.raw<int32_t>(2);
  w.u8(T_TUPLE);
  w.u8((uint8_t)nfields);
  for (int i = 0; i < nfields; ++i) w.symbol(fields[i].name);
  w.counter++;  // the Tuple{...} DataType of the field types
  w.u8(T_DATATYPE);
  w.symbol("Tuple");
  w.module_core();
  w.raw<int32_t>(nfields);
  for (int i = 0; i < nfields; ++i) w.field_type(fields[i]);
  // the field values
  int rc = R2M_OK;
  for (int i = 0; i < nfields && w.ok && rc == R2M_OK; ++i) {
    const r2m_jl_field &fl = fields[i];
    switch (fl.kind) {
      case R2M_JL_INT: w.int64(fl.ival); break;
      case R2M_JL_BOOL: w.u8(fl.ival ? T_TRUE : T_FALSE); break;
      case R2M_JL_STRING: w.string(fl.str, (size_t)fl.str_len); break;
      case R2M_JL_ARRAY: {
        w.counter++;
        w.u8(T_ARRAY);
        if (fl.elty != R2M_JL_U8) w.elty(fl.elty);
        if (fl.ndims == 1) {
          w.int64(fl.dims[0]);
        } else {
          w.u8(T_TUPLE);
          w.u8(2);
          w.int64(fl.dims[0]);
          w.int64(fl.dims[1]);
        }
        const size_t n = (size_t)fl.dims[0] * (fl.ndims == 2 ? (size_t)fl.dims[1] : 1);
        w.bytes(fl.data, n * (size_t)jl_elem_size(fl.elty));
        break;
      }
      case R2M_JL_STRVEC: {
        w.counter++;
        w.u8(T_ARRAY);
        w.elty(100);
        w.int64(fl.dims[0]);
        const int32_t *idx = static_cast<const int32_t *>(fl.data);
        for (int64_t e = 0; e < fl.dims[0]; ++e) {
          const int32_t u = idx[e];
          if (u < 0 || u >= fl.nuniq) {
            rc = r2m::fail(R2M_EINVAL, std::string("string index out of range in ") + fl.name);
            break;
          }
          const int64_t a = fl.uniq_off[u], b = fl.uniq_off[u + 1];
          if (a < 0 || b < a || b - a > INT32_MAX) {
            rc = r2m::fail(R2M_EINVAL, std::string("bad string offsets in ") + fl.name);
            break;
          }
          w.string(fl.blob + a, (size_t)(b - a));
        }
        break;
      }
      default: break;
    }
  }
  const bool ok = w.ok;
  if (fclose(f) != 0 && rc == R2M_OK && ok) return r2m::fail(R2M_EIO, std::string("cannot write ") + path);
  if (rc) return rc;
  if (!ok) return r2m::fail(R2M_EIO, std::string("cannot write ") + path);
  return R2M_OK;
}
