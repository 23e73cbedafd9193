// meshio.cu -- OFELI's XML mesh files (".m"): Mesh::get and Mesh::put on the
// host, and the hand-off of a P1 mesh read from a file to the device path
// (ofg_mesh_create: device pattern, colouring, assembly).
//
// Reading restates what OFELI's XMLParser does with a mesh file:
//   Mesh::get                src/mesh/Mesh.cpp:2639-2668
//   XMLParser::on_tag_open   src/io/XMLParser.cpp:646-760
//   XMLParser::read_mesh     src/io/XMLParser.cpp:1174-1217 (Mesh / Elements / Sides attributes)
//   XMLParser::on_cdata      src/io/XMLParser.cpp:1316-1335 (whitespace tokens)
//   XMLParser::read_mesh_data src/io/XMLParser.cpp:2211-2295 (Nodes / Elements / Sides records)
//   DOFCode                  src/mesh/MeshUtil.cpp:101-116
// and writing restates Mesh::put (src/mesh/Mesh.cpp:2731-2806).  Properties
// kept because OFELI has them:
//   * a coordinate is converted by std::stof, so it is the nearest float to
//     the decimal text, stored as a double;
//   * a node or side mark is split into one code per DOF by DOFCode, whose
//     sign handling yields the digits of |mark| for a negative mark;
//   * every tag opening resets the element node count, so an Elements block
//     needs its nodes attribute; the Mesh tag sets shape defaults from the
//     dimension known before each of its attributes (attributes in name
//     order);
//   * the Material block's (code, name) pairs are registered in order, then
//     every element code not yet registered as "Generic" (Material::set /
//     check, src/mesh/Material.cpp:90-125); the Material tag also switches
//     the parser to material properties, so no mesh data after it is read;
//   * put writes a negative node mark and a negative side code as the 64-bit
//     unsigned wrap-around (OFELI multiplies a size_t by the sign), and an
//     empty Material block whenever the material registered under code 1 is
//     not "Generic" (a mesh read from a file counts no materials of its own,
//     so the block never lists any).
// Where OFELI's behaviour is undefined (a record cut short at the end of a
// block, an element naming a node that does not exist, more nodes per record
// than its fixed arrays hold) the reader reports OFG_ERR_ARG instead; so it
// does for a second Nodes, Elements or Sides text (another block, or one
// split by a comment), where OFELI restarts its labels and later sorts by
// them.
//
// The Nodes / Elements / Sides text is converted by a team of host threads:
// the block is cut into chunks at whitespace, each chunk counts its tokens, a
// prefix sum gives every chunk its first token number (hence record and
// field), and each chunk converts its tokens straight into the arrays.
// put formats record ranges in parallel and writes them in order.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.cuh"

struct ofg_mesh_file {
   int dim = 2, nb_dof = 1;
   int el_shape = 0, el_nodes = 0;    // OFELI shape code, nodes per element
   int sd_shape = 0, sd_nodes = 0;
   int64_t nn = 0, ne = 0, ns = 0;
   std::vector<double> coords;        // nn * dim
   std::vector<int32_t> node_code;    // nn * nb_dof
   std::vector<int32_t> elem;         // ne * el_nodes, 0-based node indices
   std::vector<int32_t> elem_code;    // ne
   std::vector<int32_t> side;         // ns * sd_nodes, 0-based
   std::vector<int32_t> side_code;    // ns * nb_dof
   std::vector<std::pair<int32_t, std::string>> materials;   // the Material block's pairs
};

namespace {

using ofg::Error;
using ofg::guarded;

int g_threads = 0;   // 0: all hardware threads

// OFELI's element shape codes (include/OFELI_Config.h:274-282) and the names
// Mesh::put writes for codes 0..7.
const char* const kPutShape[8] = {"none", "point", "line", "triangle", "quadrilateral",
                                  "tetrahedron", "hexahedron", "pentahedron"};
enum { SH_NONE = 0, SH_POINT = 1, SH_LINE = 2, SH_TRIANGLE = 3, SH_QUAD = 4, SH_TETRA = 5,
       SH_HEXA = 6, SH_PENTA = 7, SH_PRISM = 8, SH_PYRAMID = 9 };
constexpr int kMaxNbDof = 6;        // MAX_NBDOF_NODE / MAX_NBDOF_SIDE
constexpr int kMaxElNodes = 20;     // read_mesh_data's nnd[20]
constexpr int kMaxSdNodes = 8;      // read_mesh_data's nnd[8]

// Element(label, shape string, code): the ElStSh map of src/mesh/Element.cpp
// :43-56 (an unknown name maps to 0).
int element_shape(const std::string& s)
{
   static const std::map<std::string, int> m = {
       {"point", SH_POINT},      {"line", SH_LINE},          {"triangle", SH_TRIANGLE},
       {"tria", SH_TRIANGLE},    {"quadrilateral", SH_QUAD}, {"quad", SH_QUAD},
       {"tetrahedron", SH_TETRA}, {"tetra", SH_TETRA},       {"hexahedron", SH_HEXA},
       {"hexa", SH_HEXA},        {"pentahedron", SH_PENTA},  {"penta", SH_PENTA},
       {"prism", SH_PRISM},      {"pyramid", SH_PYRAMID}};
   auto it = m.find(s);
   return it == m.end() ? SH_NONE : it->second;
}

// Side::shape_index (src/mesh/Side.cpp:360-368); other names leave OFELI's
// shape unset, an error here.
int side_shape(const std::string& s)
{
   if (s == "line") return SH_LINE;
   if (s == "tria" || s == "triangle") return SH_TRIANGLE;
   if (s == "quad" || s == "quadrilateral") return SH_QUAD;
   throw Error(OFG_ERR_ARG, "unknown side shape \"" + s + "\"");
}

inline bool is_space(char c)
{
   return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

int team_size(size_t bytes)
{
   int hw = (int)std::thread::hardware_concurrency();
   int t = g_threads > 0 ? g_threads : std::max(1, hw);
   int by_size = (int)std::max<size_t>(1, bytes >> 18);   // at least 256 KiB per thread
   return std::max(1, std::min({t, by_size, 256}));
}

// f(t) for t in [0, T) on T threads; the first exception is rethrown.
template <class F>
void parallel_for(int T, F&& f)
{
   if (T <= 1) {
      f(0);
      return;
   }
   std::vector<std::exception_ptr> err(T);
   std::vector<std::thread> th;
   th.reserve(T - 1);
   for (int t = 1; t < T; ++t)
      th.emplace_back([&, t] {
         try { f(t); } catch (...) { err[t] = std::current_exception(); }
      });
   try { f(0); } catch (...) { err[0] = std::current_exception(); }
   for (auto& x : th) x.join();
   for (auto& e : err)
      if (e) std::rethrow_exception(e);
}

// std::stoi of one token: leading blanks, optional sign, decimal digits,
// stop at the first other character; no digit or a value outside int fails.
inline int32_t to_int(const char* p, const char* e, const char* what)
{
   while (p < e && is_space(*p)) ++p;
   bool neg = false;
   if (p < e && (*p == '+' || *p == '-')) neg = *p++ == '-';
   const char* d = p;
   uint64_t v = 0;
   while (p < e && *p >= '0' && *p <= '9') {
      if (v > 1000000000000ull) throw Error(OFG_ERR_ARG, std::string(what) + " out of int range");
      v = v * 10 + uint64_t(*p - '0');
      ++p;
   }
   if (p == d) throw Error(OFG_ERR_ARG, std::string("invalid ") + what + " token");
   if (v > (neg ? 2147483648ull : 2147483647ull))
      throw Error(OFG_ERR_ARG, std::string(what) + " out of int range");
   return neg ? int32_t(-int64_t(v)) : int32_t(v);
}

// std::stof of one token (strtof, then out_of_range on ERANGE).  Normal
// non-zero results come from std::from_chars (correctly rounded like
// strtof); signs, hexadecimal, zero, subnormal, infinite and NaN forms go
// through strtof itself so that its errno behaviour is kept.  The token is
// followed by whitespace, '<' or the buffer's terminating NUL, where strtof
// stops.
inline double to_coord(const char* p, const char* e)
{
   float v = 0.f;
   auto r = std::from_chars(p, e, v);
   if (r.ec == std::errc() && std::isnormal(v)) return double(v);
   errno = 0;
   char* end = nullptr;
   float w = std::strtof(p, &end);
   if (end == p) throw Error(OFG_ERR_ARG, "invalid coordinate token");
   if (errno == ERANGE) throw Error(OFG_ERR_ARG, "coordinate out of float range");
   return double(w);
}

// DOFCode (src/mesh/MeshUtil.cpp:101-116): mark -> one code per DOF, most
// significant digit first; the running remainder keeps the mark's sign and
// each quotient is multiplied by it, so a negative mark gives |digits|.
inline void dof_code(int32_t mark, int nb_dof, int32_t* code)
{
   if (mark == INT32_MIN) throw Error(OFG_ERR_ARG, "code out of range");
   int64_t j = mark;
   int64_t sign = mark < 0 ? -1 : 1;
   for (int k = 0; k < nb_dof; ++k) {
      int64_t kk = 1;
      for (int q = 0; q < nb_dof - k - 1; ++q) kk *= 10;
      int64_t m = j / kk;
      code[k] = int32_t(m * sign);
      j -= m * kk;
   }
}

// The text of one block, cut into chunks for a team of threads, with the
// number of whitespace-delimited tokens before each chunk.
struct Block {
   std::vector<const char*> cut;
   std::vector<int64_t> first;   // first[t] = tokens in chunks before t; first[T] = all
   int T = 1;

   Block(const char* s, const char* e, const char* what)
   {
      size_t bytes = size_t(e - s);
      T = team_size(bytes);
      cut.assign(T + 1, s);
      cut[T] = e;
      for (int t = 1; t < T; ++t) {
         const char* c = std::max(s + bytes * size_t(t) / size_t(T), cut[t - 1]);
         while (c < e && !is_space(*c)) ++c;   // never split a token
         cut[t] = c;
      }
      first.assign(T + 1, 0);
      parallel_for(T, [&](int t) {
         int64_t n = 0;
         bool in = false;
         for (const char* p = cut[t]; p < cut[t + 1]; ++p) {
            char c = *p;
            if (c == '&' || c == '>')
               throw Error(OFG_ERR_ARG, std::string("unexpected '") + c + "' in " + what + " data");
            bool sp = is_space(c);
            n += (!sp && !in);
            in = !sp;
         }
         first[t + 1] = n;
      });
      for (int t = 0; t < T; ++t) first[t + 1] += first[t];
   }

   int64_t records(int rec, const char* what) const
   {
      if (first[T] % rec) throw Error(OFG_ERR_ARG, std::string(what) + " block ends inside a record");
      return first[T] / rec;
   }

   // visit(record, field, token begin, token end) for every token
   template <class Visit>
   void convert(int rec, Visit&& visit) const
   {
      parallel_for(T, [&](int t) {
         int64_t g = first[t];
         const char* p = cut[t];
         const char* end = cut[t + 1];
         while (true) {
            while (p < end && is_space(*p)) ++p;
            if (p >= end) break;
            const char* q = p;
            while (q < end && !is_space(*q)) ++q;
            visit(g / rec, int(g % rec), p, q);
            ++g;
            p = q;
         }
      });
   }
};

struct Reader {
   ofg_mesh_file* f;
   bool set_mesh = true;      // XMLParser::_set_mesh
   bool mesh_type = true;     // XMLParser::_type == EType::MESH
   std::string tag;           // XMLParser::_tag_name: the last opened tag
   std::string el_shape = "triangle", sd_shape = "line";
   int el_nodes = 0, sd_nodes = 2;
   bool have_nodes = false, have_elements = false, have_sides = false;
   // device reading: data blocks are recorded here instead of converted
   struct Deferred {
      int kind;   // 0 Nodes, 1 Elements, 2 Sides
      const char* s;
      const char* e;
      int per;    // nodes per element / side
   };
   std::vector<Deferred>* defer = nullptr;
   bool defer_fallback = false;   // a layout the device reader leaves to the host reader

   void open(const std::string& name, const std::map<std::string, std::string>& attrs)
   {
      el_nodes = 0;
      tag = name;
      if (name == "Material") mesh_type = false;
      if (!(set_mesh && mesh_type)) return;
      for (const auto& a : attrs) {
         if (name == "Mesh") {
            if (f->dim == 1) el_shape = "line";
            else if (f->dim == 2) el_shape = "triangle", sd_shape = "line", sd_nodes = 2;
            else if (f->dim == 3) el_shape = "tetrahedron", sd_shape = "triangle", sd_nodes = 3;
            if (a.first == "file")
               throw Error(OFG_ERR_ARG, "mesh files that include another file are not supported");
            else if (a.first == "dim")
               f->dim = to_int(a.second.data(), a.second.data() + a.second.size(), "dim");
            else if (a.first == "nb_dof")
               f->nb_dof = to_int(a.second.data(), a.second.data() + a.second.size(), "nb_dof");
         }
         else if (name == "Elements" || name == "elements") {
            if (a.first == "shape") el_shape = a.second;
            if (a.first == "nodes")
               el_nodes = to_int(a.second.data(), a.second.data() + a.second.size(), "nodes");
         }
         else if (name == "Sides" || name == "sides") {
            if (a.first == "shape") sd_shape = a.second;
            if (a.first == "nodes")
               sd_nodes = to_int(a.second.data(), a.second.data() + a.second.size(), "nodes");
         }
      }
   }

   void close(const std::string& name)
   {
      if (name == "Mesh") set_mesh = false;
   }

   void check_dims()
   {
      OFG_REQUIRE(f->dim >= 1 && f->dim <= 3, OFG_ERR_ARG, "mesh dim must be 1, 2 or 3");
      OFG_REQUIRE(f->nb_dof >= 1 && f->nb_dof <= kMaxNbDof, OFG_ERR_ARG, "nb_dof must be 1..6");
   }

   static bool data_tag(const std::string& t)
   {
      return t == "Nodes" || t == "nodes" || t == "Elements" || t == "elements" || t == "Sides" ||
             t == "sides";
   }

   void text(const char* s, const char* e)
   {
      // data blocks check for '>' while they are tokenised
      if (!(set_mesh && mesh_type && data_tag(tag)) && memchr(s, '>', size_t(e - s)))
         throw Error(OFG_ERR_ARG, "XML: unexpected character '>' in text");
      if (tag == "Material" && set_mesh) {
         material(s, e);
         return;
      }
      if (!(set_mesh && mesh_type)) return;
      if (tag == "Nodes" || tag == "nodes") nodes(s, e);
      else if (tag == "Elements" || tag == "elements") elements(s, e);
      else if (tag == "Sides" || tag == "sides") sides(s, e);
   }

   // (code, name) pairs, each registered as Material::set does
   void material(const char* s, const char* e)
   {
      std::vector<std::pair<const char*, const char*>> tok;
      for (const char* p = s; p < e;) {
         while (p < e && is_space(*p)) ++p;
         if (p >= e) break;
         const char* q = p;
         while (q < e && !is_space(*q)) ++q;
         tok.emplace_back(p, q);
         p = q;
      }
      OFG_REQUIRE(tok.size() % 2 == 0, OFG_ERR_ARG, "Material block ends inside a (code, name) pair");
      for (size_t i = 0; i < tok.size(); i += 2)
         f->materials.emplace_back(to_int(tok[i].first, tok[i].second, "material code"),
                                   std::string(tok[i + 1].first, tok[i + 1].second));
   }

   void nodes(const char* s, const char* e)
   {
      check_dims();
      OFG_REQUIRE(!have_nodes, OFG_ERR_ARG, "more than one Nodes text");
      if (defer && (have_elements || have_sides)) defer_fallback = true;
      OFG_REQUIRE(f->ne == 0 && f->ns == 0, OFG_ERR_ARG, "Nodes must come before Elements and Sides");
      have_nodes = true;
      if (defer) {
         defer->push_back({0, s, e, 0});
         return;
      }
      const int dim = f->dim, nd = f->nb_dof, rec = dim + 1;
      Block blk(s, e, "Nodes");
      const int64_t n = blk.records(rec, "Nodes");
      f->coords.resize(size_t(n) * dim);
      f->node_code.resize(size_t(n) * nd);
      double* X = f->coords.data();
      int32_t* C = f->node_code.data();
      blk.convert(rec, [&](int64_t r, int fld, const char* p, const char* q) {
         if (fld < dim) X[r * dim + fld] = to_coord(p, q);
         else dof_code(to_int(p, q, "node code"), nd, C + r * nd);
      });
      f->nn = n;
   }

   void elements(const char* s, const char* e)
   {
      check_dims();
      OFG_REQUIRE(el_nodes >= 1 && el_nodes <= kMaxElNodes, OFG_ERR_ARG,
                  "Elements needs a nodes attribute between 1 and 20");
      OFG_REQUIRE(!have_elements, OFG_ERR_ARG, "more than one Elements text");
      int shape = element_shape(el_shape);
      have_elements = true;
      f->el_shape = shape;
      f->el_nodes = el_nodes;
      if (defer) {
         defer->push_back({1, s, e, el_nodes});
         return;
      }
      const int k = el_nodes, rec = k + 1;
      const int64_t nn = f->nn;
      Block blk(s, e, "Elements");
      const int64_t n = blk.records(rec, "Elements");
      f->elem.resize(size_t(n) * k);
      f->elem_code.resize(size_t(n));
      int32_t* E = f->elem.data();
      int32_t* C = f->elem_code.data();
      blk.convert(rec, [&](int64_t r, int fld, const char* p, const char* q) {
         int32_t v = to_int(p, q, fld < k ? "element node" : "element code");
         if (fld < k) {
            if (v < 1 || v > nn) throw Error(OFG_ERR_ARG, "element names a node that does not exist");
            E[r * k + fld] = v - 1;
         }
         else C[r] = v;
      });
      f->ne = n;
   }

   void sides(const char* s, const char* e)
   {
      check_dims();
      OFG_REQUIRE(sd_nodes >= 1 && sd_nodes <= kMaxSdNodes, OFG_ERR_ARG,
                  "Sides needs between 1 and 8 nodes per side");
      OFG_REQUIRE(!have_sides, OFG_ERR_ARG, "more than one Sides text");
      int shape = side_shape(sd_shape);
      have_sides = true;
      f->sd_shape = shape;
      f->sd_nodes = sd_nodes;
      if (defer) {
         defer->push_back({2, s, e, sd_nodes});
         return;
      }
      const int k = sd_nodes, rec = k + 1, nd = f->nb_dof;
      const int64_t nn = f->nn;
      Block blk(s, e, "Sides");
      const int64_t n = blk.records(rec, "Sides");
      f->side.resize(size_t(n) * k);
      f->side_code.resize(size_t(n) * nd);
      int32_t* S = f->side.data();
      int32_t* C = f->side_code.data();
      blk.convert(rec, [&](int64_t r, int fld, const char* p, const char* q) {
         int32_t v = to_int(p, q, fld < k ? "side node" : "side code");
         if (fld < k) {
            if (v < 1 || v > nn) throw Error(OFG_ERR_ARG, "side names a node that does not exist");
            S[r * k + fld] = v - 1;
         }
         else dof_code(v, nd, C + r * nd);
      });
      f->ns = n;
   }
};

inline bool is_label(char c)
{
   return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || (c >= '0' && c <= '9') || c == '_' ||
          c == '-' || c == ':' || c == '.';
}

// memchr, with the bytes beyond the first MiB searched by a team of threads
// (the end of a large data block).
const char* find_char(const char* p, const char* e, char c)
{
   size_t n = size_t(e - p), head = size_t(1) << 20;
   if (n <= head) return (const char*)memchr(p, c, n);
   if (const char* q = (const char*)memchr(p, c, head)) return q;
   const char* s = p + head;
   size_t rest = size_t(e - s);
   int T = team_size(rest);
   std::vector<const char*> hit(T, nullptr);
   parallel_for(T, [&](int t) {
      size_t a = rest * size_t(t) / size_t(T), z = rest * size_t(t + 1) / size_t(T);
      hit[t] = (const char*)memchr(s + a, c, z - a);
   });
   for (const char* h : hit)
      if (h) return h;
   return nullptr;
}

// xmlsp's blanks between and inside tags (a CR reads as a newline there).
inline bool tag_space(char c) { return c == ' ' || c == '\n' || c == '\t' || c == '\r'; }

// The XML grammar of xmlsp (src/io/xmlsp/xmlsp.cpp:100-450), which OFELI's
// mesh reader runs on the whole file: blanks and '<' only outside the root;
// "<?...?>" only outside the root; "<!--...-->" anywhere; "<![CDATA[...]]>"
// inside elements; "<!DOCTYPE ...>" before the root; a tag name and attribute
// names of [A-Za-z0-9_.:-]; attributes written name="value" with no blank
// around '=' and double quotes only; "/>" closes a tag at once; "</name>"
// with no blank must match the open tag; '>' may not appear in text.  Text
// between tags is delivered when it holds a character other than a blank.
// Entity references are refused in data blocks and attribute values.
void scan_xml(const char* b, const char* e, Reader& rd)
{
   std::vector<std::string> stack;
   bool had_root = false;   // set when a root element was a single tag (as xmlsp does)
   const char* p = b;
   auto fail = [](const std::string& m) { throw Error(OFG_ERR_ARG, "XML: " + m); };
   auto find = [&](const char* from, const char* pat) -> const char* {
      size_t n = strlen(pat);
      for (const char* q = from; q + n <= e; ++q) {
         q = (const char*)memchr(q, pat[0], size_t(e - q));
         if (!q || q + n > e) return nullptr;
         if (!memcmp(q, pat, n)) return q;
      }
      return nullptr;
   };
   auto label = [&]() {
      const char* n0 = p;
      while (p < e && is_label(*p)) ++p;
      return std::string(n0, p);
   };
   while (p < e) {
      if (stack.empty()) {
         while (p < e && tag_space(*p)) ++p;
         if (p >= e) break;
         if (*p != '<') fail("unexpected character outside tag");
      }
      else {
         const char* lt = find_char(p, e, '<');
         const char* te = lt ? lt : e;
         if (te > p) {
            bool blank = true;
            for (const char* q = p; q < te && blank; ++q) blank = tag_space(*q);
            if (!blank) rd.text(p, te);
         }
         if (!lt) fail("open tag missing close tag");
         p = lt;
      }
      ++p;   // past '<'
      if (p >= e) fail("tag not finished");
      if (*p == '?') {
         if (!stack.empty()) fail("processing instruction inside an element");
         const char* q = find(p, "?>");
         if (!q) fail("processing instruction not closed");
         p = q + 2;
         continue;
      }
      if (*p == '!') {
         ++p;
         if (p < e && *p == '-') {
            if (p + 1 >= e || p[1] != '-') fail("unexpected character, expecting '-' for comment");
            const char* q = find(p, "-->");   // "<!-->" already closes
            if (!q) fail("comment not closed");
            p = q + 3;
         }
         else if (p < e && *p == '[') {
            if (e - p < 7 || memcmp(p, "[CDATA[", 7)) fail("unknown element");
            const char* q = find(p + 7, "]]>");
            if (!q) fail("CDATA not closed");
            if (stack.empty()) fail("CDATA outside the root element");
            bool blank = true;
            for (const char* c = p + 7; c < q && blank; ++c) blank = tag_space(*c);
            if (!blank) rd.text(p + 7, q);
            p = q + 3;
         }
         else {
            if (!stack.empty() || had_root) fail("unexpected character, expected comment or DOCTYPE");
            if (e - p < 7 || memcmp(p, "DOCTYPE", 7)) fail("unknown element");
            const char* q = (const char*)memchr(p, '>', size_t(e - p));
            if (!q) fail("DOCTYPE not closed");
            if (q - p < 8) fail("unknown element");
            p = q + 1;
         }
         continue;
      }
      if (*p == '/') {
         ++p;
         std::string name = label();
         if (p >= e || *p != '>') fail("unexpected character in closing tag");
         if (stack.empty() || stack.back() != name) fail("closing tag '" + name + "' does not match");
         rd.close(name);
         stack.pop_back();
         ++p;
         continue;
      }
      if (!is_label(*p)) fail("unexpected character at the beginning of a tag");
      if (stack.empty() && had_root) fail("a second root tag found");
      std::string name = label();
      std::map<std::string, std::string> attrs;
      bool single = false;
      bool after_name = true;
      while (true) {
         if (p >= e) fail("tag not finished");
         char c = *p;
         if (tag_space(c)) {
            ++p;
            after_name = false;
         }
         else if (c == '>') {
            ++p;
            break;
         }
         else if (c == '/') {
            if (p + 1 >= e || p[1] != '>') fail("unexpected character in tag level after slash");
            p += 2;
            single = true;
            break;
         }
         else if (is_label(c) && !after_name) {
            std::string key = label();
            if (p >= e || *p != '=') fail("unexpected character in attribute name");
            if (p + 1 >= e || p[1] != '"') fail("unexpected character, expected double quote");
            p += 2;
            const char* v1 = (const char*)memchr(p, '"', size_t(e - p));
            if (!v1) fail("tag not finished");
            if (memchr(p, '&', size_t(v1 - p))) fail("entity references in attribute values are not supported");
            attrs[key] = std::string(p, v1);
            p = v1 + 1;
         }
         else
            fail("unexpected character in tag");
      }
      rd.open(name, attrs);
      if (single) {
         rd.close(name);
         if (stack.empty()) had_root = true;
      }
      else
         stack.push_back(name);
   }
   if (!stack.empty()) fail("open tag missing close tag");
}

// Whole file into memory (parallel reads for large files), NUL-terminated.
std::unique_ptr<char[]> slurp(const char* path, size_t& size)
{
   int fd = ::open(path, O_RDONLY);
   if (fd < 0) throw Error(OFG_ERR_ARG, std::string("cannot open ") + path);
   struct stat st;
   if (fstat(fd, &st) != 0) {
      ::close(fd);
      throw Error(OFG_ERR_ARG, std::string("cannot stat ") + path);
   }
   size = size_t(st.st_size);
   std::unique_ptr<char[]> buf(new char[size + 1]);
   int T = team_size(size >> 2);
   try {
      parallel_for(T, [&](int t) {
         size_t a = size * size_t(t) / size_t(T), z = size * size_t(t + 1) / size_t(T);
         while (a < z) {
            ssize_t r = ::pread(fd, buf.get() + a, z - a, off_t(a));
            if (r <= 0) throw Error(OFG_ERR_ARG, std::string("read error on ") + path);
            a += size_t(r);
         }
      });
   }
   catch (...) {
      ::close(fd);
      throw;
   }
   ::close(fd);
   buf[size] = 0;
   return buf;
}

// ------------------------------------------------------------------ put --
template <class Fmt>
void put_records(FILE* fp, int64_t n, Fmt&& fmt)
{
   if (n <= 0) return;
   int T = team_size(size_t(n) * 32);
   std::vector<std::string> out(T);
   parallel_for(T, [&](int t) {
      int64_t a = n * t / T, z = n * (t + 1) / T;
      std::string& s = out[t];
      s.reserve(size_t(z - a) * 64);
      char line[512];
      for (int64_t r = a; r < z; ++r) {
         int len = fmt(r, line);
         s.append(line, size_t(len));
      }
   });
   for (auto& s : out)
      if (fwrite(s.data(), 1, s.size(), fp) != s.size())
         throw Error(OFG_ERR_ARG, "write error");
}

uint64_t pow10u(int k)
{
   uint64_t v = 1;
   while (k-- > 0) v *= 10;
   return v;
}

// Material::getName(1) after Mesh::get: the file's pairs first, then
// Material::check registering each unseen element code as "Generic"; " "
// when code 1 is not registered.
std::string material_name_1(const ofg_mesh_file* f)
{
   for (const auto& m : f->materials)
      if (m.first == 1) return m.second;
   for (int64_t i = 0; i < f->ne; ++i)
      if (f->elem_code[size_t(i)] == 1) return "Generic";
   return " ";
}

void put_file(const ofg_mesh_file* f, const char* path)
{
   OFG_REQUIRE(f->el_shape >= 0 && f->el_shape < 8, OFG_ERR_ARG,
               "Mesh::put has no name for prism or pyramid elements");
   FILE* fp = fopen(path, "wb");
   if (!fp) throw Error(OFG_ERR_ARG, std::string("cannot create ") + path);
   try {
      const int n = f->nb_dof, dim = f->dim;
      fprintf(fp, "<?xml version=\"1.0\"?>\n<OFELI_File>\n<info>\n   <title></title>\n"
                  "   <date></date>\n   <author></author>\n</info>\n");
      fprintf(fp, "<Mesh dim=\"%d\" nb_dof=\"%d\">\n", dim, n);
      if (f->nn > 0) {
         fputs("   <Nodes>\n", fp);
         put_records(fp, f->nn, [&](int64_t r, char* line) {
            int len = 0;
            for (int i = 0; i < dim; ++i)
               len += snprintf(line + len, 64, "  %18.8e", f->coords[size_t(r) * dim + i]);
            const int32_t* c = f->node_code.data() + size_t(r) * n;
            uint64_t m = 0;
            for (int j = 0; j < n; ++j) m += uint64_t(c[j] < 0 ? -int64_t(c[j]) : c[j]) * pow10u(n - 1 - j);
            if (c[0] < 0) m = 0 - m;
            len += snprintf(line + len, 64, "%10llu\n", (unsigned long long)m);
            return len;
         });
         fputs("   </Nodes>\n", fp);
      }
      if (f->ne > 0) {
         fprintf(fp, "   <Elements shape=\"%s\" nodes=\"%d\">\n", kPutShape[f->el_shape], f->el_nodes);
         const int k = f->el_nodes;
         put_records(fp, f->ne, [&](int64_t r, char* line) {
            int len = 0;
            for (int i = 0; i < k; ++i)
               len += snprintf(line + len, 32, "%8lld", (long long)f->elem[size_t(r) * k + i] + 1);
            len += snprintf(line + len, 32, "%8d\n", f->elem_code[size_t(r)]);
            return len;
         });
         fputs("   </Elements>\n", fp);
      }
      if (f->ns > 0) {
         fprintf(fp, "   <Sides shape=\"%s\" nodes=\"%d\">\n", kPutShape[f->sd_shape], f->sd_nodes);
         const int k = f->sd_nodes;
         put_records(fp, f->ns, [&](int64_t r, char* line) {
            int len = 0;
            for (int i = 0; i < k; ++i)
               len += snprintf(line + len, 32, "%8lld", (long long)f->side[size_t(r) * k + i] + 1);
            uint64_t m = 0;
            for (int j = 0; j < n; ++j)
               m += uint64_t(int64_t(f->side_code[size_t(r) * n + j])) * pow10u(n - 1 - j);
            len += snprintf(line + len, 32, "%6llu\n", (unsigned long long)m);
            return len;
         });
         fputs("   </Sides>\n", fp);
      }
      if (material_name_1(f) != "Generic") fputs("   <Material>\n   </Material>\n", fp);
      fputs("</Mesh>\n</OFELI_File>\n", fp);
      if (fflush(fp) != 0) throw Error(OFG_ERR_ARG, "write error");
   }
   catch (...) {
      fclose(fp);
      throw;
   }
   if (fclose(fp) != 0) throw Error(OFG_ERR_ARG, "write error");
}

}  // namespace

namespace {

using namespace ofg;

// ------------------------------------------------------ device reading --
// ofg_mesh_read: the file's bytes are read into a pinned staging buffer and
// copied to the device once, piece by piece as they are read; the host walks
// the XML structure (tags are few)
// and the Nodes / Elements / Sides texts are tokenised and converted by
// kernels, straight into the device mesh's buffers.
//
// Tokenising: a 256-thread block covers a 4 KiB tile, one 16-byte aligned
// load per thread; a byte starts a token when it is not blank and the byte
// before it is (or the block starts there).  Pass 1 counts starts per tile,
// a scan gives each tile its first token number, pass 2 recounts, scans the
// threads' counts inside the block and converts every token it starts
// (record = token / fields, field = token % fields).
//
// Coordinates: the token's decimal mantissa (up to 19 significant digits)
// and exponent are parsed exactly; when the mantissa is below 2^53 and the
// decimal exponent within +-22, M * 10^e (or M / 10^-e) is one correctly
// rounded double operation, and rounding that double to float gives strtof's
// result unless the double lies exactly on a float rounding midpoint.  Every
// other token (a sign '+', hexadecimal, infinity, NaN, more digits, a wider
// exponent, a midpoint, a result outside the normal float range) is listed
// and converted on the host by the same conversion as ofg_mesh_file_read,
// which also raises the errors std::stof would.  Integers convert exactly on
// the device.  Errors are flagged by kind; the host reports them.

constexpr int kParseThreads = 256;
constexpr int kParseChunk = 16;
constexpr int64_t kParseTile = kParseThreads * kParseChunk;
enum : unsigned { PF_CHAR = 1, PF_INT = 2, PF_RANGE = 4, PF_LABEL = 8, PF_CODE = 16, PF_FULL = 32 };

__device__ __forceinline__ bool dev_space(unsigned c) { return c == 32u || (c >= 9u && c <= 13u); }

// Start bits of the 16 aligned bytes at a0 (positions outside [beg, end)
// read as blanks).
__device__ __forceinline__ unsigned token_starts(const char* buf, int64_t beg, int64_t end,
                                                 int64_t a0, bool& bad)
{
   if (a0 >= end) return 0;
   const uint4 w = *reinterpret_cast<const uint4*>(buf + a0);
   const uint32_t word[4] = {w.x, w.y, w.z, w.w};
   bool prev = (a0 - 1 < beg) ? true : dev_space((unsigned char)buf[a0 - 1]);
   unsigned bits = 0;
#pragma unroll
   for (int i = 0; i < kParseChunk; ++i) {
      const unsigned c = (word[i >> 2] >> (8 * (i & 3))) & 0xffu;
      const int64_t q = a0 + i;
      const bool inside = q >= beg && q < end;
      const bool sp = !inside || dev_space(c);
      bad |= inside && (c == '&' || c == '>');
      if (!sp && prev) bits |= 1u << i;
      prev = sp;
   }
   return bits;
}

__global__ void __launch_bounds__(kParseThreads) parse_count(const char* buf, int64_t beg, int64_t end,
                                                             int64_t base, int64_t* tile_count,
                                                             unsigned* flags)
{
   __shared__ int warp_sum[kParseThreads / 32];
   const int64_t a0 = base + (int64_t)blockIdx.x * kParseTile + (int64_t)threadIdx.x * kParseChunk;
   bool bad = false;
   int n = __popc(token_starts(buf, beg, end, a0, bad));
   if (bad) atomicOr(flags, PF_CHAR);
#pragma unroll
   for (int o = 16; o; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
   if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = n;
   __syncthreads();
   if (threadIdx.x == 0) {
      int t = 0;
      for (int w = 0; w < kParseThreads / 32; ++w) t += warp_sum[w];
      tile_count[blockIdx.x] = t;
   }
}

// std::stoi of the token [p, q) (see to_int); 0 ok, else a PF_ kind.
__device__ __forceinline__ unsigned dev_int(const char* buf, int64_t p, int64_t q, int32_t& v)
{
   bool neg = false;
   if (p < q && (buf[p] == '+' || buf[p] == '-')) neg = buf[p++] == '-';
   const int64_t d = p;
   uint64_t x = 0;
   while (p < q && buf[p] >= '0' && buf[p] <= '9') {
      if (x > 1000000000000ull) return PF_RANGE;
      x = x * 10 + uint64_t(buf[p] - '0');
      ++p;
   }
   if (p == d) return PF_INT;
   if (x > (neg ? 2147483648ull : 2147483647ull)) return PF_RANGE;
   v = neg ? int32_t(-int64_t(x)) : int32_t(x);
   return 0;
}

__constant__ double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,
                                  1e8,  1e9,  1e10, 1e11, 1e12, 1e13, 1e14, 1e15,
                                  1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};

// std::stof of the token [p, q) when the fast path above decides it; false
// sends the token to the host.
__device__ __forceinline__ bool dev_coord(const char* buf, int64_t p, int64_t q, double& v)
{
   bool neg = false;
   if (p < q && buf[p] == '-') neg = true, ++p;
   if (p + 1 < q && buf[p] == '0' && (buf[p + 1] == 'x' || buf[p + 1] == 'X')) return false;
   uint64_t M = 0;
   int nd = 0, dexp = 0;
   bool any = false, lost = false;
   while (p < q && buf[p] >= '0' && buf[p] <= '9') {
      const int dg = buf[p++] - '0';
      any = true;
      if (M == 0 && dg == 0) continue;
      if (nd < 19) M = M * 10 + uint64_t(dg), ++nd;
      else ++dexp, lost |= dg != 0;
   }
   if (p < q && buf[p] == '.') {
      ++p;
      while (p < q && buf[p] >= '0' && buf[p] <= '9') {
         const int dg = buf[p++] - '0';
         any = true;
         if (M == 0 && dg == 0) {
            --dexp;
            continue;
         }
         if (nd < 19) M = M * 10 + uint64_t(dg), ++nd, --dexp;
         else lost |= dg != 0;
      }
   }
   if (!any || lost) return false;
   if (p < q && (buf[p] == 'e' || buf[p] == 'E')) {
      int64_t j = p + 1;
      bool eneg = false;
      if (j < q && (buf[j] == '+' || buf[j] == '-')) eneg = buf[j++] == '-';
      if (j < q && buf[j] >= '0' && buf[j] <= '9') {
         int x = 0;
         while (j < q && buf[j] >= '0' && buf[j] <= '9') {
            if (x < 100000) x = x * 10 + (buf[j] - '0');
            ++j;
         }
         dexp += eneg ? -x : x;
      }
   }
   if (M == 0) {
      v = neg ? -0.0 : 0.0;
      return true;
   }
   if (M > (uint64_t(1) << 53) || dexp < -22 || dexp > 22) return false;
   double d = dexp >= 0 ? __dmul_rn(double(M), kPow10[dexp]) : __ddiv_rn(double(M), kPow10[-dexp]);
   if (!(d >= 1.1754943508222875e-38 && d <= 3.4028234663852886e38)) return false;
   const float f = __double2float_rn(d);
   const double fd = double(f);
   if (fd != d) {
      const int nb = __float_as_int(f) + (d > fd ? 1 : -1);   // the float neighbour on d's side
      const double mid = 0.5 * (fd + double(__int_as_float(nb)));
      if (mid == d) return false;
   }
   v = neg ? -fd : fd;
   return true;
}

struct ParseOut {
   int kind;              // 0 Nodes, 1 Elements, 2 Sides
   int fields;            // tokens per record
   int dim;               // Nodes: coordinates per record
   int64_t nn;            // Elements / Sides: node labels must be in 1..nn
   double* coords;        // Nodes
   int32_t* code;         // Nodes (nb_dof 1: DOFCode gives |mark|)
   int32_t* elem;         // Elements (0-based)
   int64_t* fb_pos;       // coordinate tokens left to the host
   int64_t* fb_out;
   int fb_cap;
   int* fb_count;
};

__global__ void __launch_bounds__(kParseThreads) parse_convert(const char* buf, int64_t beg, int64_t end,
                                                               int64_t base, const int64_t* tile_off,
                                                               ParseOut o, unsigned* flags)
{
   __shared__ int warp_sum[kParseThreads / 32];
   const int64_t a0 = base + (int64_t)blockIdx.x * kParseTile + (int64_t)threadIdx.x * kParseChunk;
   bool bad = false;
   unsigned bits = token_starts(buf, beg, end, a0, bad);
   const int n = __popc(bits);
   // exclusive scan of the threads' counts
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   int incl = n;
#pragma unroll
   for (int k = 1; k < 32; k <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, k);
      if (lane >= k) incl += y;
   }
   if (lane == 31) warp_sum[warp] = incl;
   __syncthreads();
   int before = 0;
   for (int w = 0; w < warp; ++w) before += warp_sum[w];
   int64_t g = tile_off[blockIdx.x] + before + incl - n;
   unsigned err = 0;
   while (bits) {
      const int i = __ffs(bits) - 1;
      bits &= bits - 1;
      const int64_t p = a0 + i;
      int64_t q = p;
      while (q < end && !dev_space((unsigned char)buf[q])) ++q;
      const int64_t r = g / o.fields;
      const int fld = int(g - r * o.fields);
      ++g;
      if (o.kind == 0 && fld < o.dim) {
         double x;
         if (dev_coord(buf, p, q, x))
            o.coords[r * o.dim + fld] = x;
         else {
            const int slot = atomicAdd(o.fb_count, 1);
            if (slot < o.fb_cap) {
               o.fb_pos[slot] = p;
               o.fb_out[slot] = r * o.dim + fld;
            }
            else
               err |= PF_FULL;
         }
         continue;
      }
      int32_t v = 0;
      const unsigned st = dev_int(buf, p, q, v);
      if (st) {
         err |= st;
         continue;
      }
      if (o.kind == 0) {   // node mark, nb_dof 1
         if (v == INT32_MIN) err |= PF_CODE;
         else o.code[r] = v < 0 ? -v : v;
      }
      else if (fld < o.fields - 1) {   // a node label
         if (v < 1 || v > o.nn) err |= PF_LABEL;
         else if (o.kind == 1) o.elem[r * (o.fields - 1) + fld] = v - 1;
      }
      else if (o.kind == 2 && v == INT32_MIN)
         err |= PF_CODE;
   }
   if (bad) err |= PF_CHAR;
   if (err) atomicOr(flags, err);
}

__global__ void scatter_values(int n, const int64_t* idx, const double* val, double* out)
{
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i < n) out[idx[i]] = val[i];
}

// The pinned staging buffer, kept between reads (grown on demand).
std::mutex g_pin_mu;
char* g_pin = nullptr;
size_t g_pin_cap = 0;

char* pinned_staging(size_t n)
{
   if (n > g_pin_cap) {
      if (g_pin) OFG_CUDA(cudaFreeHost(g_pin));
      g_pin = nullptr;
      g_pin_cap = 0;
      OFG_CUDA(cudaHostAlloc((void**)&g_pin, n, cudaHostAllocDefault));
      g_pin_cap = n;
   }
   return g_pin;
}

}  // namespace

void ofg::meshio_release_staging()
{
   std::lock_guard<std::mutex> lock(g_pin_mu);
   if (g_pin) cudaFreeHost(g_pin);
   g_pin = nullptr;
   g_pin_cap = 0;
}

namespace {

// The file into the staging buffer by a team of threads, NUL-terminated,
// and on to the device: each thread copies every piece it has read (4 MiB at
// most) to `db` at once, so the transfer overlaps the reading.
size_t read_to_device(const char* path, char*& buf, DBuf<char>& db)
{
   int fd = ::open(path, O_RDONLY);
   if (fd < 0) throw Error(OFG_ERR_ARG, std::string("cannot open ") + path);
   struct stat st;
   if (fstat(fd, &st) != 0) {
      ::close(fd);
      throw Error(OFG_ERR_ARG, std::string("cannot stat ") + path);
   }
   const size_t size = size_t(st.st_size);
   try {
      buf = pinned_staging(size + 1);
      db.alloc(((size + 15) & ~size_t(15)) + 32);
      int device = 0;
      OFG_CUDA(cudaGetDevice(&device));
      const cudaStream_t st_ = stream();
      constexpr size_t kPiece = size_t(4) << 20;
      int T = team_size(size >> 2);
      parallel_for(T, [&](int t) {
         OFG_CUDA(cudaSetDevice(device));
         size_t a = size * size_t(t) / size_t(T);
         const size_t z = size * size_t(t + 1) / size_t(T);
         while (a < z) {
            const size_t e = std::min(z, a + kPiece);
            size_t p = a;
            while (p < e) {
               ssize_t r = ::pread(fd, buf + p, e - p, off_t(p));
               if (r <= 0) throw Error(OFG_ERR_ARG, std::string("read error on ") + path);
               p += size_t(r);
            }
            OFG_CUDA(cudaMemcpyAsync(db.p + a, buf + a, e - a, cudaMemcpyHostToDevice, st_));
            a = e;
         }
      });
   }
   catch (...) {
      ::close(fd);
      throw;
   }
   ::close(fd);
   buf[size] = 0;
   return size;
}

// Tokens of one block: tile counts and their exclusive scan; returns the total.
int64_t count_tokens(const char* dbuf, int64_t beg, int64_t end, int64_t& base, int64_t& tiles,
                     DBuf<int64_t>& off, unsigned* dflags)
{
   base = beg & ~int64_t(15);
   tiles = (end - base + kParseTile - 1) / kParseTile;
   DBuf<int64_t> cnt(tiles + 1);
   off.alloc(tiles + 1);
   OFG_CUDA(cudaMemsetAsync(cnt.p + tiles, 0, sizeof(int64_t), stream()));
   parse_count<<<(unsigned)tiles, kParseThreads, 0, stream()>>>(dbuf, beg, end, base, cnt.p, dflags);
   count_launch();
   OFG_LAUNCH_CHECK();
   scan_exclusive_i64(cnt.p, off.p, tiles + 1);
   int64_t total = 0;
   OFG_CUDA(cudaMemcpyAsync(&total, off.p + tiles, sizeof(int64_t), cudaMemcpyDeviceToHost, stream()));
   OFG_CUDA(cudaStreamSynchronize(stream()));
   return total;
}

void raise_parse_flags(unsigned fl)
{
   if (fl & PF_CHAR) throw Error(OFG_ERR_ARG, "unexpected '&' or '>' in mesh data");
   if (fl & PF_INT) throw Error(OFG_ERR_ARG, "invalid integer token in mesh data");
   if (fl & PF_RANGE) throw Error(OFG_ERR_ARG, "integer out of int range in mesh data");
   if (fl & PF_CODE) throw Error(OFG_ERR_ARG, "code out of range");
   if (fl & PF_LABEL) throw Error(OFG_ERR_ARG, "element or side names a node that does not exist");
}

// Mesh(file, true) on the device; false when the layout is left to the host
// reader (blocks out of order, too many coordinates for the device path).
bool read_device(const char* path, ofg_mesh** out)
{
   std::lock_guard<std::mutex> lock(g_pin_mu);
   char* hb = nullptr;
   DBuf<char> db;
   const size_t size = read_to_device(path, hb, db);
   ofg_mesh_file meta;
   Reader rd{&meta};
   std::vector<Reader::Deferred> blocks;
   rd.defer = &blocks;
   scan_xml(hb, hb + size, rd);
   if (rd.defer_fallback) return false;
   OFG_REQUIRE((meta.dim == 2 && meta.el_shape == SH_TRIANGLE && meta.el_nodes == 3) ||
                   (meta.dim == 3 && meta.el_shape == SH_TETRA && meta.el_nodes == 4),
               OFG_ERR_ARG, "the P1 path takes triangles in 2-D or tetrahedra in 3-D");
   OFG_REQUIRE(meta.nb_dof == 1, OFG_ERR_ARG, "the P1 path takes meshes with one DOF per node");
   DBuf<unsigned> dflags(1);
   dflags.zero();
   struct Counted {
      const Reader::Deferred* d;
      int64_t beg, end, base, tiles, ntok;
      DBuf<int64_t> off;
   };
   std::vector<Counted> cb(blocks.size());
   int64_t nn = 0, ne = 0;
   for (size_t i = 0; i < blocks.size(); ++i) {
      Counted& c = cb[i];
      c.d = &blocks[i];
      c.beg = blocks[i].s - hb;
      c.end = blocks[i].e - hb;
      c.ntok = count_tokens(db.p, c.beg, c.end, c.base, c.tiles, c.off, dflags.p);
      const int fields = c.d->kind == 0 ? meta.dim + 1 : c.d->per + 1;
      const char* what = c.d->kind == 0 ? "Nodes" : c.d->kind == 1 ? "Elements" : "Sides";
      if (c.ntok % fields) throw Error(OFG_ERR_ARG, std::string(what) + " block ends inside a record");
      if (c.d->kind == 0) nn = c.ntok / fields;
      if (c.d->kind == 1) ne = c.ntok / fields;
   }
   OFG_REQUIRE(nn > 0 && ne > 0, OFG_ERR_ARG, "bad mesh arguments");
   OFG_REQUIRE(ne * (meta.dim + 1) < (int64_t(1) << 31) && nn < (int64_t(1) << 31), OFG_ERR_SIZE,
               "mesh too large");
   std::unique_ptr<ofg_mesh> m(new_mesh(meta.dim, nn, ne));
   const int fb_cap = int(std::min<int64_t>(nn * meta.dim, 1 << 20));
   DBuf<int64_t> fb_pos(fb_cap), fb_out(fb_cap);
   DBuf<int> fb_count(1);
   fb_count.zero();
   for (Counted& c : cb) {
      if (c.tiles == 0) continue;
      ParseOut o{};
      o.kind = c.d->kind;
      o.fields = c.d->kind == 0 ? meta.dim + 1 : c.d->per + 1;
      o.dim = meta.dim;
      o.nn = nn;
      o.coords = m->coords.p;
      o.code = m->code.p;
      o.elem = m->elem.p;
      o.fb_pos = fb_pos.p;
      o.fb_out = fb_out.p;
      o.fb_cap = fb_cap;
      o.fb_count = fb_count.p;
      parse_convert<<<(unsigned)c.tiles, kParseThreads, 0, stream()>>>(db.p, c.beg, c.end, c.base,
                                                                       c.off.p, o, dflags.p);
      count_launch();
      OFG_LAUNCH_CHECK();
   }
   unsigned fl = 0;
   int nfb = 0;
   OFG_CUDA(cudaMemcpyAsync(&fl, dflags.p, sizeof(unsigned), cudaMemcpyDeviceToHost, stream()));
   OFG_CUDA(cudaMemcpyAsync(&nfb, fb_count.p, sizeof(int), cudaMemcpyDeviceToHost, stream()));
   OFG_CUDA(cudaStreamSynchronize(stream()));
   raise_parse_flags(fl);
   if (fl & PF_FULL) return false;
   if (nfb > 0) {
      std::vector<int64_t> pos = fb_pos.to_host(nfb);
      std::vector<double> val(nfb);
      for (int i = 0; i < nfb; ++i) {
         const char* p = hb + pos[i];
         const char* q = p;
         while (q < hb + size && !is_space(*q)) ++q;
         val[i] = to_coord(p, q);
      }
      DBuf<double> dval(nfb);
      dval.upload(val.data(), nfb);
      scatter_values<<<(nfb + 255) / 256, 256, 0, stream()>>>(nfb, fb_out.p, dval.p, m->coords.p);
      count_launch();
      OFG_LAUNCH_CHECK();
      OFG_CUDA(cudaStreamSynchronize(stream()));   // val is a pageable source
   }
   finish_mesh(m.get());
   *out = m.release();
   return true;
}

}  // namespace

extern "C" {

int ofg_mesh_file_set_threads(int n)
{
   return guarded("ofg_mesh_file_set_threads", [&] {
      OFG_REQUIRE(n >= 0, OFG_ERR_ARG, "thread count must be >= 0");
      g_threads = n;
   });
}

int ofg_mesh_file_read(const char* path, ofg_mesh_file** out)
{
   return guarded("ofg_mesh_file_read", [&] {
      OFG_REQUIRE(path && out, OFG_ERR_ARG, "null argument");
      size_t size = 0;
      std::unique_ptr<char[]> buf = slurp(path, size);
      std::unique_ptr<ofg_mesh_file> f(new ofg_mesh_file());
      Reader rd{f.get()};
      scan_xml(buf.get(), buf.get() + size, rd);
      *out = f.release();
   });
}

int ofg_mesh_file_create(int dim, int nb_dof, int64_t nn, const double* coords,
                         const int32_t* node_code, int el_shape, int el_nodes, int64_t ne,
                         const int32_t* elem, const int32_t* elem_code, int sd_shape, int sd_nodes,
                         int64_t ns, const int32_t* sides, const int32_t* side_code,
                         ofg_mesh_file** out)
{
   return guarded("ofg_mesh_file_create", [&] {
      OFG_REQUIRE(out && dim >= 1 && dim <= 3 && nb_dof >= 1 && nb_dof <= kMaxNbDof && nn >= 0 &&
                      ne >= 0 && ns >= 0,
                  OFG_ERR_ARG, "bad mesh sizes");
      OFG_REQUIRE(nn == 0 || (coords && node_code), OFG_ERR_ARG, "null node arrays");
      OFG_REQUIRE(ne == 0 || (elem && elem_code && el_nodes >= 1 && el_nodes <= kMaxElNodes &&
                              el_shape >= 0 && el_shape <= SH_PYRAMID),
                  OFG_ERR_ARG, "bad element arrays");
      OFG_REQUIRE(ns == 0 || (sides && side_code && sd_nodes >= 1 && sd_nodes <= kMaxSdNodes &&
                              (sd_shape == SH_LINE || sd_shape == SH_TRIANGLE || sd_shape == SH_QUAD)),
                  OFG_ERR_ARG, "bad side arrays");
      std::unique_ptr<ofg_mesh_file> f(new ofg_mesh_file());
      f->dim = dim, f->nb_dof = nb_dof, f->nn = nn, f->ne = ne, f->ns = ns;
      f->el_shape = ne ? el_shape : 0, f->el_nodes = ne ? el_nodes : 0;
      f->sd_shape = ns ? sd_shape : 0, f->sd_nodes = ns ? sd_nodes : 0;
      f->coords.assign(coords, coords + nn * dim);
      f->node_code.assign(node_code, node_code + nn * nb_dof);
      if (ne) {
         f->elem.assign(elem, elem + ne * el_nodes);
         f->elem_code.assign(elem_code, elem_code + ne);
         for (int32_t v : f->elem)
            OFG_REQUIRE(v >= 0 && v < nn, OFG_ERR_ARG, "element names a node that does not exist");
      }
      if (ns) {
         f->side.assign(sides, sides + ns * sd_nodes);
         f->side_code.assign(side_code, side_code + ns * nb_dof);
         for (int32_t v : f->side)
            OFG_REQUIRE(v >= 0 && v < nn, OFG_ERR_ARG, "side names a node that does not exist");
      }
      *out = f.release();
   });
}

int ofg_mesh_file_from_mesh(const ofg_mesh* m, ofg_mesh_file** out)
{
   return guarded("ofg_mesh_file_from_mesh", [&] {
      OFG_REQUIRE(m && out, OFG_ERR_ARG, "null argument");
      int dim = 0;
      int64_t nn = 0, ne = 0;
      OFG_REQUIRE(ofg_mesh_info(m, &dim, &nn, &ne, nullptr) == OFG_OK, OFG_ERR_ARG,
                  ofg_last_error());
      std::unique_ptr<ofg_mesh_file> f(new ofg_mesh_file());
      f->dim = dim, f->nb_dof = 1, f->nn = nn, f->ne = ne;
      f->el_shape = dim == 2 ? SH_TRIANGLE : SH_TETRA, f->el_nodes = dim + 1;
      f->coords.resize(size_t(nn) * dim);
      f->node_code.resize(size_t(nn));
      f->elem.resize(size_t(ne) * (dim + 1));
      f->elem_code.assign(size_t(ne), 1);
      int rc = ofg_mesh_get(m, f->coords.data(), f->elem.data(), f->node_code.data(), nullptr);
      if (rc != OFG_OK) throw Error(rc, ofg_last_error());
      if (m->rect_nx >= 0) {
         // Mesh(xmin,...,cx0,cxN,cy0,cyN) adds a LINE side with code -c along
         // every boundary line whose code c is negative (src/mesh/Mesh.cpp
         // :623-672), in the order x = xmin, x = xmax, y = ymin, y = ymax
         const int64_t nx = m->rect_nx, ny = m->rect_ny;
         auto add = [&](int64_t a, int64_t b, int c) {
            f->side.push_back(int32_t(a - 1));
            f->side.push_back(int32_t(b - 1));
            f->side_code.push_back(-c);
         };
         const int* c = m->rect_code;
         if (c[0] < 0)
            for (int64_t j = 1, n = 1; j <= ny; ++j, ++n) add(n, n + 1, c[0]);
         if (c[1] < 0)
            for (int64_t j = 1, n = nx * (ny + 1) + 1; j <= ny; ++j, ++n) add(n, n + 1, c[1]);
         if (c[2] < 0)
            for (int64_t i = 1, n = 1; i <= nx; ++i, n += ny + 1) add(n, n + ny + 1, c[2]);
         if (c[3] < 0)
            for (int64_t i = 1, n = ny + 1; i <= nx; ++i, n += ny + 1) add(n, n + ny + 1, c[3]);
         f->ns = int64_t(f->side_code.size());
         if (f->ns) f->sd_shape = SH_LINE, f->sd_nodes = 2;
      }
      *out = f.release();
   });
}

int ofg_mesh_file_info(const ofg_mesh_file* f, int* dim, int* nb_dof, int64_t* nn, int* el_shape,
                       int* el_nodes, int64_t* ne, int* sd_shape, int* sd_nodes, int64_t* ns)
{
   return guarded("ofg_mesh_file_info", [&] {
      OFG_REQUIRE(f, OFG_ERR_ARG, "null mesh file");
      if (dim) *dim = f->dim;
      if (nb_dof) *nb_dof = f->nb_dof;
      if (nn) *nn = f->nn;
      if (el_shape) *el_shape = f->el_shape;
      if (el_nodes) *el_nodes = f->el_nodes;
      if (ne) *ne = f->ne;
      if (sd_shape) *sd_shape = f->sd_shape;
      if (sd_nodes) *sd_nodes = f->sd_nodes;
      if (ns) *ns = f->ns;
   });
}

int ofg_mesh_file_get(const ofg_mesh_file* f, double* coords, int32_t* node_code, int32_t* elem,
                      int32_t* elem_code, int32_t* sides, int32_t* side_code)
{
   return guarded("ofg_mesh_file_get", [&] {
      OFG_REQUIRE(f, OFG_ERR_ARG, "null mesh file");
      auto cp = [](auto* dst, const auto& v) {
         if (dst && !v.empty()) memcpy(dst, v.data(), v.size() * sizeof(v[0]));
      };
      cp(coords, f->coords);
      cp(node_code, f->node_code);
      cp(elem, f->elem);
      cp(elem_code, f->elem_code);
      cp(sides, f->side);
      cp(side_code, f->side_code);
   });
}

int ofg_mesh_file_write(const ofg_mesh_file* f, const char* path)
{
   return guarded("ofg_mesh_file_write", [&] {
      OFG_REQUIRE(f && path, OFG_ERR_ARG, "null argument");
      put_file(f, path);
   });
}

int ofg_mesh_file_destroy(ofg_mesh_file* f)
{
   return guarded("ofg_mesh_file_destroy", [&] { delete f; });
}

int ofg_mesh_read(const char* path, ofg_mesh** out)
{
   return guarded("ofg_mesh_read", [&] {
      OFG_REQUIRE(path && out, OFG_ERR_ARG, "null argument");
      if (read_device(path, out)) return;
      // layouts left to the host reader: read, then hand over
      ofg_mesh_file* f = nullptr;
      int rc = ofg_mesh_file_read(path, &f);
      if (rc != OFG_OK) throw Error(rc, ofg_last_error());
      std::unique_ptr<ofg_mesh_file> keep(f);
      rc = ofg_mesh_create_from_file(f, out);
      if (rc != OFG_OK) throw Error(rc, ofg_last_error());
   });
}

int ofg_mesh_create_from_file(const ofg_mesh_file* f, ofg_mesh** out)
{
   return guarded("ofg_mesh_create_from_file", [&] {
      OFG_REQUIRE(f && out, OFG_ERR_ARG, "null argument");
      OFG_REQUIRE((f->dim == 2 && f->el_shape == SH_TRIANGLE && f->el_nodes == 3) ||
                      (f->dim == 3 && f->el_shape == SH_TETRA && f->el_nodes == 4),
                  OFG_ERR_ARG, "the P1 path takes triangles in 2-D or tetrahedra in 3-D");
      OFG_REQUIRE(f->nb_dof == 1, OFG_ERR_ARG, "the P1 path takes meshes with one DOF per node");
      int rc = ofg_mesh_create(f->dim, f->nn, f->coords.data(), f->ne, f->elem.data(),
                               f->node_code.data(), out);
      if (rc != OFG_OK) throw Error(rc, ofg_last_error());
   });
}

}  // extern "C"
