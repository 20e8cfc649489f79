// ANML front-end: a small XML reader plus the VASim symbol-set grammar.
//
// Behaviour follows the reference loader:
//   * code/src/commons/NFALoader.cpp:70-154  load_nfa_from_anml (element set,
//     "automata-network" one or two levels under the root, unsupported
//     elements rejected);
//   * code/src/commons/NFALoader.cpp:24-67   start attribute and STE fields;
//   * code/src/commons/vasim_helper.cpp:40-480 parseSymbolSet (the escape,
//     range, class and inversion rules, including its quirks).
// The reference parses XML through pugixml with parse_default|parse_declaration;
// attribute values therefore get entity expansion (named and numeric, the
// latter encoded as UTF-8) and tab/CR/LF -> space conversion, which this
// reader reproduces. Unlike the reference, errors are returned, never exit().
#include "anml.h"

#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <unordered_map>

namespace ngap {

namespace {

struct XmlElem {
  std::string name;
  std::vector<std::pair<std::string, std::string>> attrs;
  std::vector<int> children;  // indices into the element arena
  bool has_text = false;      // non-whitespace character data among children
  const std::string* attr(const char* key) const {
    for (auto& kv : attrs)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
};

class XmlReader {
 public:
  XmlReader(const char* s, size_t n) : s_(s), n_(n) {}

  // Parses the whole document. Returns false and sets err on malformed XML.
  bool parse(std::vector<XmlElem>& arena, std::vector<int>& roots, std::string& err) {
    arena_ = &arena;
    std::vector<int> stack;
    while (p_ < n_) {
      if (s_[p_] != '<') {
        size_t q = p_;
        bool ws = true;
        while (q < n_ && s_[q] != '<') {
          char c = s_[q];
          if (!(c == ' ' || c == '\t' || c == '\r' || c == '\n')) ws = false;
          q++;
        }
        if (!ws && !stack.empty()) arena[stack.back()].has_text = true;
        p_ = q;
        continue;
      }
      if (starts("<!--")) {
        size_t e = find("-->", p_ + 4);
        if (e == npos) return fail(err, "unterminated comment");
        p_ = e + 3;
        continue;
      }
      if (starts("<![CDATA[")) {
        size_t e = find("]]>", p_ + 9);
        if (e == npos) return fail(err, "unterminated CDATA");
        if (e > p_ + 9 && !stack.empty()) arena[stack.back()].has_text = true;
        p_ = e + 3;
        continue;
      }
      if (starts("<?")) {
        size_t e = find("?>", p_ + 2);
        if (e == npos) return fail(err, "unterminated processing instruction");
        p_ = e + 2;
        continue;
      }
      if (starts("<!")) {  // DOCTYPE and friends: skip with bracket nesting
        int depth = 0;
        size_t q = p_ + 2;
        for (; q < n_; q++) {
          if (s_[q] == '[') depth++;
          else if (s_[q] == ']') depth--;
          else if (s_[q] == '>' && depth <= 0) break;
        }
        if (q >= n_) return fail(err, "unterminated declaration");
        p_ = q + 1;
        continue;
      }
      if (starts("</")) {
        p_ += 2;
        std::string nm = read_name();
        skip_ws();
        if (p_ >= n_ || s_[p_] != '>') return fail(err, "bad end tag");
        p_++;
        if (stack.empty() || arena[stack.back()].name != nm)
          return fail(err, "mismatched end tag </" + nm + ">");
        stack.pop_back();
        continue;
      }
      // start tag
      p_++;
      XmlElem el;
      el.name = read_name();
      if (el.name.empty()) return fail(err, "bad tag name");
      bool self_close = false;
      while (true) {
        skip_ws();
        if (p_ >= n_) return fail(err, "unterminated tag");
        if (s_[p_] == '/') {
          if (p_ + 1 < n_ && s_[p_ + 1] == '>') {
            self_close = true;
            p_ += 2;
            break;
          }
          return fail(err, "bad '/' in tag");
        }
        if (s_[p_] == '>') {
          p_++;
          break;
        }
        std::string an = read_name();
        if (an.empty()) return fail(err, "bad attribute name in <" + el.name + ">");
        skip_ws();
        if (p_ >= n_ || s_[p_] != '=') return fail(err, "attribute without value");
        p_++;
        skip_ws();
        if (p_ >= n_ || (s_[p_] != '"' && s_[p_] != '\'')) return fail(err, "unquoted attribute");
        char q = s_[p_++];
        size_t b = p_;
        while (p_ < n_ && s_[p_] != q) p_++;
        if (p_ >= n_) return fail(err, "unterminated attribute value");
        std::string raw(s_ + b, p_ - b);
        p_++;
        el.attrs.emplace_back(an, decode_attr(raw));
      }
      int idx = (int)arena.size();
      arena.push_back(std::move(el));
      if (stack.empty())
        roots.push_back(idx);
      else
        arena[stack.back()].children.push_back(idx);
      if (!self_close) stack.push_back(idx);
    }
    if (!stack.empty()) return fail(err, "unclosed element <" + arena[stack.back()].name + ">");
    return true;
  }

 private:
  static constexpr size_t npos = (size_t)-1;
  bool starts(const char* t) const {
    size_t l = strlen(t);
    return p_ + l <= n_ && memcmp(s_ + p_, t, l) == 0;
  }
  size_t find(const char* t, size_t from) const {
    size_t l = strlen(t);
    for (size_t i = from; i + l <= n_; i++)
      if (memcmp(s_ + i, t, l) == 0) return i;
    return npos;
  }
  void skip_ws() {
    while (p_ < n_ && (s_[p_] == ' ' || s_[p_] == '\t' || s_[p_] == '\r' || s_[p_] == '\n')) p_++;
  }
  std::string read_name() {
    size_t b = p_;
    while (p_ < n_) {
      char c = s_[p_];
      if (c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '>' || c == '/' || c == '=' ||
          c == '<')
        break;
      p_++;
    }
    return std::string(s_ + b, p_ - b);
  }
  static void put_utf8(std::string& o, uint32_t cp) {
    if (cp < 0x80) {
      o.push_back((char)cp);
    } else if (cp < 0x800) {
      o.push_back((char)(0xC0 | (cp >> 6)));
      o.push_back((char)(0x80 | (cp & 0x3F)));
    } else if (cp < 0x10000) {
      o.push_back((char)(0xE0 | (cp >> 12)));
      o.push_back((char)(0x80 | ((cp >> 6) & 0x3F)));
      o.push_back((char)(0x80 | (cp & 0x3F)));
    } else {
      o.push_back((char)(0xF0 | (cp >> 18)));
      o.push_back((char)(0x80 | ((cp >> 12) & 0x3F)));
      o.push_back((char)(0x80 | ((cp >> 6) & 0x3F)));
      o.push_back((char)(0x80 | (cp & 0x3F)));
    }
  }
  // Entity expansion and whitespace conversion of an attribute value.
  static std::string decode_attr(const std::string& r) {
    std::string o;
    o.reserve(r.size());
    for (size_t i = 0; i < r.size(); i++) {
      char c = r[i];
      if (c == '\r') {  // end-of-line normalisation: CR LF -> one space
        o.push_back(' ');
        if (i + 1 < r.size() && r[i + 1] == '\n') i++;
        continue;
      }
      if (c == '\t' || c == '\n') {
        o.push_back(' ');
        continue;
      }
      if (c != '&') {
        o.push_back(c);
        continue;
      }
      size_t semi = r.find(';', i);
      if (semi == std::string::npos) {
        o.push_back(c);
        continue;
      }
      std::string ent = r.substr(i + 1, semi - i - 1);
      if (ent == "lt") o.push_back('<');
      else if (ent == "gt") o.push_back('>');
      else if (ent == "amp") o.push_back('&');
      else if (ent == "quot") o.push_back('"');
      else if (ent == "apos") o.push_back('\'');
      else if (ent.size() > 1 && ent[0] == '#') {
        char* endp = nullptr;
        unsigned long cp = (ent[1] == 'x' || ent[1] == 'X') ? strtoul(ent.c_str() + 2, &endp, 16)
                                                            : strtoul(ent.c_str() + 1, &endp, 10);
        put_utf8(o, (uint32_t)cp);
      } else {
        o.append(r, i, semi - i + 1);  // unknown entity: keep verbatim
      }
      i = semi;
    }
    return o;
  }
  bool fail(std::string& err, const std::string& m) {
    err = m;
    return false;
  }

  const char* s_;
  size_t n_;
  size_t p_ = 0;
  std::vector<XmlElem>* arena_ = nullptr;
};

void set_range(Bits256& col, int start, int end) {
  for (; start <= end; start++) col.set(start);
}

}  // namespace

bool parse_symbol_set(const std::string& ss, Bits256& col, std::string& err) {
  col = Bits256();
  if (ss == "*") {
    col.set_all();
    return true;
  }
  if (ss == ".") {  // apcompile reads "." as "^\x0a"
    col.set_all();
    col.reset('\n');
    return true;
  }
  if (!ss.empty() && ss.front() == '{' && ss.back() == '}') {
    err = "curly-brace symbol sets are not supported: " + ss;
    return false;
  }
  const uint32_t kOpenBracket = 256;
  bool escaped = false, inverting = false, range_set = false;
  int bracket_sem = 0;
  uint32_t last_char = 0, range_start = 0;
  auto put = [&](uint32_t ch) {
    col.set((int)ch);
    if (range_set) {
      set_range(col, (int)range_start, (int)ch);
      range_set = false;
    }
    last_char = ch;
  };
  auto at = [&](size_t i) -> char { return i < ss.size() ? ss[i] : '\0'; };
  size_t index = 0;
  while (index < ss.size()) {
    unsigned char c = (unsigned char)ss[index];
    switch (c) {
      case '[':
        if (escaped) {
          put(c);
          escaped = false;
        } else {
          last_char = kOpenBracket;
          bracket_sem++;
        }
        break;
      case ']':
        if (escaped) {
          put(c);
          escaped = false;
        } else {
          bracket_sem--;
        }
        break;
      case '{':
      case '}':  // literal either way; an escape before it stays pending
        put(c);
        break;
      case '\\':
        if (escaped) {
          put(c);
          escaped = false;
        } else {
          escaped = true;
        }
        break;
      case 'n': case 'r': case 't': case 'a': case 'b': case 'f': case 'v': case '\'': case '"': {
        if (escaped) {
          uint32_t m = c;
          switch (c) {
            case 'n': m = '\n'; break;
            case 'r': m = '\r'; break;
            case 't': m = '\t'; break;
            case 'a': m = '\a'; break;
            case 'b': m = '\b'; break;
            case 'f': m = '\f'; break;
            case 'v': m = '\v'; break;
            default: break;
          }
          put(m);
          escaped = false;
        } else {
          put(c);
        }
        break;
      }
      case '-':
        if (escaped || last_char == kOpenBracket) {
          put('-');
          escaped = false;
        } else {
          range_set = true;
          range_start = last_char;
        }
        break;
      case 's':
        if (escaped) {  // whitespace class; no range or last_char update
          col.set('\n');
          col.set('\t');
          col.set('\r');
          col.set(0x0B);
          col.set(0x0C);
          col.set(0x20);
          escaped = false;
        } else {
          put(c);
        }
        break;
      case 'd':
        if (escaped) {
          set_range(col, 48, 57);
          escaped = false;
        } else {
          put(c);
        }
        break;
      case 'w':
        if (escaped) {
          col.set('_');
          set_range(col, 48, 57);
          set_range(col, 65, 90);
          set_range(col, 97, 122);
          escaped = false;
        } else {
          put(c);
        }
        break;
      case '^':
        if (escaped) {
          put(c);
          escaped = false;
        } else {
          inverting = true;
        }
        break;
      case 'x':
        if (escaped) {
          ++index;
          char hex[3] = {at(index), at(index + 1), '\0'};
          unsigned char number = (unsigned char)strtoul(hex, nullptr, 16);
          ++index;
          put(number);
          escaped = false;
        } else {
          put(c);
        }
        break;
      default:
        escaped = false;  // an escape of an ordinary character is dropped
        put(c);
        break;
    }
    index++;
  }
  if (inverting) col.flip();
  if (bracket_sem != 0) {
    err = "malformed brackets in symbol set: " + ss;
    return false;
  }
  return true;
}

namespace {

int start_kind(const std::string* s) {
  if (!s) return kStartNone;
  if (*s == "start-of-data") return kStartOfData;
  if (*s == "all-input") return kStartAllInput;
  return kStartNone;
}

}  // namespace

int parse_anml(const char* xml, size_t len, AnmlNfa& out) {
  std::vector<XmlElem> arena;
  std::vector<int> roots;
  std::string err;
  XmlReader rd(xml, len);
  if (!rd.parse(arena, roots, err)) {
    set_error("ANML parse error: %s", err.c_str());
    return NGAP_E_PARSE;
  }
  auto child = [&](int parent, const char* nm) -> int {
    const std::vector<int>& ch = parent < 0 ? roots : arena[parent].children;
    for (int c : ch)
      if (arena[c].name == nm) return c;
    return -1;
  };
  int net = -1;
  int anml = child(-1, "anml");
  if (anml >= 0) net = child(anml, "automata-network");
  if (net < 0) net = child(-1, "automata-network");
  if (net < 0) {
    set_error("ANML parse error: no automata-network element");
    return NGAP_E_PARSE;
  }
  if (arena[net].has_text) {
    set_error("ANML parse error: character data inside automata-network is not supported");
    return NGAP_E_PARSE;
  }
  out = AnmlNfa();
  std::unordered_map<std::string, int> ids;
  std::vector<std::vector<std::string>> targets;
  for (int c : arena[net].children) {
    const XmlElem& e = arena[c];
    if (e.name == "state-transition-element") {
      AnmlNode nd;
      const std::string* id = e.attr("id");
      const std::string* sym = e.attr("symbol-set");
      nd.str_id = id ? *id : std::string();
      nd.symbol_set_str = sym ? *sym : std::string();
      nd.start = (uint8_t)start_kind(e.attr("start"));
      if (!parse_symbol_set(nd.symbol_set_str, nd.symbols, err)) {
        set_error("ANML parse error in STE '%s': %s", nd.str_id.c_str(), err.c_str());
        return NGAP_E_PARSE;
      }
      if (ids.count(nd.str_id)) {
        set_error("ANML parse error: duplicate STE id '%s'", nd.str_id.c_str());
        return NGAP_E_PARSE;
      }
      std::vector<std::string> tg;
      for (int cc : e.children) {
        const XmlElem& ch = arena[cc];
        if (ch.name == "activate-on-match") {
          const std::string* t = ch.attr("element");
          tg.push_back(t ? *t : std::string());
        } else if (ch.name == "report-on-match") {
          nd.report = true;
          const std::string* rc = ch.attr("reportcode");
          nd.report_code = rc ? *rc : std::string();
        }
      }
      ids[nd.str_id] = (int)out.nodes.size();
      out.nodes.push_back(std::move(nd));
      targets.push_back(std::move(tg));
    } else if (e.name == "description") {
      // ignored, as in the reference
    } else {
      set_error("ANML parse error: element <%s> is not supported", e.name.c_str());
      return NGAP_E_PARSE;
    }
  }
  if (out.nodes.empty()) {
    set_error("ANML parse error: the automata-network has no state-transition-element");
    return NGAP_E_PARSE;
  }
  // Edges are keyed by id and deduplicated on insert (NFA.cpp:125-134).
  out.adj.assign(out.nodes.size(), {});
  for (size_t i = 0; i < targets.size(); i++) {
    for (auto& t : targets[i]) {
      auto it = ids.find(t);
      if (it == ids.end()) {
        set_error("ANML parse error: STE '%s' activates unknown element '%s'",
                  out.nodes[i].str_id.c_str(), t.c_str());
        return NGAP_E_PARSE;
      }
      int to = it->second;
      bool dup = false;
      for (int x : out.adj[i])
        if (x == to) dup = true;
      if (!dup) out.adj[i].push_back(to);
    }
  }
  return NGAP_OK;
}

int load_anml_file(const char* path, AnmlNfa& out) {
  std::string p(path ? path : "");
  if (p.size() < 5 || p.compare(p.size() - 5, 5, ".anml") != 0) {
    set_error("unsupported NFA file type: %s", p.c_str());
    return NGAP_E_UNSUPPORTED;
  }
  std::ifstream f(p, std::ios::binary);
  if (!f) {
    set_error("could not load .xml file: %s", p.c_str());
    return NGAP_E_IO;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  std::string s = ss.str();
  return parse_anml(s.data(), s.size(), out);
}

}  // namespace ngap
