// xml_reader.cpp -- see xml_reader.hpp.
#include "xml_reader.hpp"

#include <cctype>
#include <fstream>
#include <sstream>

namespace gdem {

namespace {

struct Parser {
  std::string const& s;
  size_t p = 0;
  explicit Parser(std::string const& str) : s(str) {}

  [[noreturn]] void fail(std::string const& what) {
    size_t line = 1;
    for (size_t i = 0; i < p && i < s.size(); ++i) line += s[i] == '\n';
    throw std::runtime_error("XML parse error line " + std::to_string(line) + ": " + what);
  }
  bool starts(const char* t) const { return s.compare(p, std::char_traits<char>::length(t), t) == 0; }
  void skipWs() { while (p < s.size() && std::isspace((unsigned char)s[p])) ++p; }
  void skipPast(const char* t) {
    size_t q = s.find(t, p);
    if (q == std::string::npos) fail(std::string("unterminated construct, expected ") + t);
    p = q + std::char_traits<char>::length(t);
  }
  // Skips <?...?>, <!--...-->, <!DOCTYPE ...> (with an optional [...] subset)
  bool skipMisc() {
    if (starts("<?")) { skipPast("?>"); return true; }
    if (starts("<!--")) { skipPast("-->"); return true; }
    if (starts("<!DOCTYPE") || starts("<!doctype")) {
      int depth = 0;
      for (; p < s.size(); ++p) {
        if (s[p] == '[') ++depth;
        else if (s[p] == ']') --depth;
        else if (s[p] == '>' && depth == 0) { ++p; return true; }
      }
      fail("unterminated DOCTYPE");
    }
    return false;
  }
  std::string name() {
    size_t b = p;
    while (p < s.size() && (std::isalnum((unsigned char)s[p]) || s[p] == '_' || s[p] == '-' ||
                            s[p] == '.' || s[p] == ':'))
      ++p;
    if (b == p) fail("expected a name");
    return s.substr(b, p - b);
  }
  static std::string decode(std::string const& t) {
    std::string o;
    for (size_t i = 0; i < t.size(); ++i) {
      if (t[i] != '&') { o += t[i]; continue; }
      size_t e = t.find(';', i);
      if (e == std::string::npos) { o += t[i]; continue; }
      std::string ent = t.substr(i + 1, e - i - 1);
      if (ent == "lt") o += '<';
      else if (ent == "gt") o += '>';
      else if (ent == "amp") o += '&';
      else if (ent == "quot") o += '"';
      else if (ent == "apos") o += '\'';
      else { o += t.substr(i, e - i + 1); }
      i = e;
    }
    return o;
  }
  std::unique_ptr<XmlNode> element() {
    if (!starts("<")) fail("expected '<'");
    ++p;
    auto n = std::make_unique<XmlNode>();
    n->name = name();
    for (;;) {
      skipWs();
      if (starts("/>")) { p += 2; return n; }
      if (starts(">")) { ++p; break; }
      std::string a = name();
      skipWs();
      if (!starts("=")) fail("expected '=' after attribute " + a);
      ++p;
      skipWs();
      if (p >= s.size() || (s[p] != '"' && s[p] != '\'')) fail("expected quoted value");
      char qc = s[p++];
      size_t e = s.find(qc, p);
      if (e == std::string::npos) fail("unterminated attribute value");
      n->attrs[a] = decode(s.substr(p, e - p));
      p = e + 1;
    }
    for (;;) {
      if (p >= s.size()) fail("unterminated element <" + n->name + ">");
      if (starts("</")) {
        p += 2;
        std::string c = name();
        if (c != n->name) fail("mismatched </" + c + "> for <" + n->name + ">");
        skipWs();
        if (!starts(">")) fail("expected '>'");
        ++p;
        return n;
      }
      if (starts("<![CDATA[")) {
        p += 9;
        size_t e = s.find("]]>", p);
        if (e == std::string::npos) fail("unterminated CDATA");
        n->text += s.substr(p, e - p);
        p = e + 3;
        continue;
      }
      if (skipMisc()) continue;
      if (starts("<")) { n->children.push_back(element()); continue; }
      size_t e = s.find('<', p);
      if (e == std::string::npos) e = s.size();
      n->text += decode(s.substr(p, e - p));
      p = e;
    }
  }
  std::unique_ptr<XmlNode> document() {
    for (;;) {
      skipWs();
      if (!skipMisc()) break;
    }
    auto root = element();
    return root;
  }
};

}  // namespace

std::string XmlNode::valueS() const {
  size_t b = text.find_first_not_of(" \t\r\n");
  if (b == std::string::npos) return std::string();
  size_t e = text.find_last_not_of(" \t\r\n");
  return text.substr(b, e - b + 1);
}

std::unique_ptr<XmlNode> parseXmlString(std::string const& text) {
  Parser P(text);
  return P.document();
}

std::unique_ptr<XmlNode> parseXmlFile(std::string const& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot open XML file " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return parseXmlString(ss.str());
}

}  // namespace gdem
