// grains_shim.cpp -- implementation of the DOM and MPI stand-ins used to
// compile the Grains3D reference as the serial oracle.  TEST INFRASTRUCTURE.
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <vector>

#include "mpi.h"
#include "xercesc/grains_dom_shim.hpp"

// ------------------------------------------------------------------- MPI --
static std::vector<size_t>& derivedSizes() {
  static std::vector<size_t> v;
  return v;
}

extern "C" size_t grains_shim_type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR: case MPI_BYTE: case MPI_UNSIGNED_CHAR: case MPI_C_BOOL: case MPI_CXX_BOOL: return 1;
    case MPI_SHORT: case MPI_UNSIGNED_SHORT: return 2;
    case MPI_INT: case MPI_UNSIGNED: case MPI_FLOAT: return 4;
    case MPI_DOUBLE: case MPI_LONG: case MPI_UNSIGNED_LONG: case MPI_LONG_LONG:
    case MPI_UNSIGNED_LONG_LONG: return 8;
    default:
      if (t >= MPI_DERIVED_BASE && (size_t)(t - MPI_DERIVED_BASE) < derivedSizes().size())
        return derivedSizes()[t - MPI_DERIVED_BASE];
      return 1;
  }
}

extern "C" int grains_shim_type_register(size_t bytes) {
  derivedSizes().push_back(bytes);
  return MPI_DERIVED_BASE + (int)derivedSizes().size() - 1;
}

// ------------------------------------------------------------- strings --
XMLCh* XMLString::transcode(const char* s) {
  size_t n = std::strlen(s);
  XMLCh* o = new XMLCh[n + 1];
  for (size_t i = 0; i < n; ++i) o[i] = (XMLCh)(unsigned char)s[i];
  o[n] = 0;
  return o;
}
char* XMLString::transcode(const XMLCh* s) {
  if (!s) {
    char* o = new char[1];
    o[0] = 0;
    return o;
  }
  size_t n = 0;
  while (s[n]) ++n;
  char* o = new char[n + 1];
  for (size_t i = 0; i < n; ++i) o[i] = (char)s[i];
  o[n] = 0;
  return o;
}
void XMLString::release(char** p) { delete[] *p; *p = nullptr; }
void XMLString::release(XMLCh** p) { delete[] *p; *p = nullptr; }

static std::u16string u16(std::string const& s) {
  std::u16string o;
  for (unsigned char c : s) o.push_back((char16_t)c);
  return o;
}
static std::string u8(std::u16string const& s) {
  std::string o;
  for (char16_t c : s) o.push_back((char)c);
  return o;
}

namespace XMLUni {
const XMLCh fgDOMNamespaces[] = u"namespaces";
const XMLCh fgXercesSchema[] = u"schema";
const XMLCh fgXercesSchemaFullChecking[] = u"schema-full-checking";
const XMLCh fgDOMDatatypeNormalization[] = u"datatype-normalization";
const XMLCh fgDOMWRTFormatPrettyPrint[] = u"format-pretty-print";
const XMLCh fgDOMValidation[] = u"validation";
}  // namespace XMLUni

// ---------------------------------------------------------------- nodes --
DOMNode::DOMNode(short type) : m_type(type) {}
DOMNode::~DOMNode() {
  for (DOMNode* c : m_children) delete c;
  for (DOMNode* a : m_attrs) delete a;
  delete m_childList;
  delete m_attrMap;
}

DOMNodeList* DOMNode::getChildNodes() const {
  if (!m_childList) m_childList = new DOMNodeList(&m_children);
  return m_childList;
}

DOMNamedNodeMap* DOMNode::getAttributes() const {
  if (m_type != ELEMENT_NODE) return nullptr;
  if (!m_attrMap) m_attrMap = new DOMNamedNodeMap(&m_attrs);
  return m_attrMap;
}

DOMNode* DOMNode::cloneNode(bool deep) const {
  DOMNode* n;
  if (m_type == ELEMENT_NODE) n = new DOMElement();
  else if (m_type == TEXT_NODE) n = new DOMText();
  else if (m_type == DOCUMENT_NODE) n = new DOMDocument();
  else n = new DOMNode(m_type);
  n->m_name = m_name;
  n->m_value = m_value;
  for (DOMNode* a : m_attrs) {
    DOMNode* c = a->cloneNode(false);
    c->m_parent = n;
    n->m_attrs.push_back(c);
  }
  if (deep)
    for (DOMNode* c : m_children) n->appendChild(c->cloneNode(true));
  return n;
}

DOMNode* DOMNode::removeChild(DOMNode* old) {
  for (size_t i = 0; i < m_children.size(); ++i)
    if (m_children[i] == old) {
      m_children.erase(m_children.begin() + (long)i);
      old->m_parent = nullptr;
      return old;   // the caller owns it (Xerces semantics); it is leaked like in the reference
    }
  return nullptr;
}

DOMNode* DOMNode::appendChild(DOMNode* n) {
  n->m_parent = this;
  m_children.push_back(n);
  return n;
}

static void collect(DOMNode const* n, std::u16string const& name, std::vector<DOMNode*>& out) {
  for (DOMNode* c : n->m_children) {
    if (c->m_type == DOMNode::ELEMENT_NODE) {
      if (name == u"*" || c->m_name == name) out.push_back(c);
      collect(c, name, out);
    }
  }
}

DOMNodeList* DOMElement::getElementsByTagName(const XMLCh* name) const {
  std::vector<DOMNode*> out;
  collect(this, std::u16string(name), out);
  return new DOMNodeList(std::move(out));
}

void DOMElement::setAttribute(const XMLCh* name, const XMLCh* value) {
  for (DOMNode* a : m_attrs)
    if (a->m_name == name) { a->m_value = value; return; }
  DOMNode* a = new DOMNode(ATTRIBUTE_NODE);
  a->m_name = name;
  a->m_value = value;
  a->m_parent = this;
  m_attrs.push_back(a);
}

DOMNode* DOMNamedNodeMap::getNamedItem(const XMLCh* name) const {
  for (DOMNode* a : *m_attrs)
    if (a->m_name == name) return a;
  return nullptr;
}

DOMElement* DOMDocument::getDocumentElement() const {
  for (DOMNode* c : m_children)
    if (c->m_type == ELEMENT_NODE) return static_cast<DOMElement*>(c);
  return nullptr;
}
DOMElement* DOMDocument::createElement(const XMLCh* name) {
  DOMElement* e = new DOMElement();
  e->m_name = name;
  return e;
}
DOMText* DOMDocument::createTextNode(const XMLCh* data) {
  DOMText* t = new DOMText();
  t->m_name = u"#text";
  t->m_value = data;
  return t;
}

// --------------------------------------------------------------- parser --
namespace {

struct Parser {
  std::string const& s;
  size_t p = 0;
  explicit Parser(std::string const& str) : s(str) {}
  bool starts(const char* t) const { return s.compare(p, std::strlen(t), t) == 0; }
  void skipPast(const char* t) {
    size_t q = s.find(t, p);
    if (q == std::string::npos) throw std::runtime_error("unterminated XML construct");
    p = q + std::strlen(t);
  }
  bool skipMisc() {
    if (starts("<?")) { skipPast("?>"); return true; }
    if (starts("<!--")) { skipPast("-->"); return true; }
    if (starts("<!DOCTYPE")) {
      int depth = 0;
      for (; p < s.size(); ++p) {
        if (s[p] == '[') ++depth;
        else if (s[p] == ']') --depth;
        else if (s[p] == '>' && depth == 0) { ++p; return true; }
      }
      throw std::runtime_error("unterminated DOCTYPE");
    }
    return false;
  }
  std::string name() {
    size_t b = p;
    while (p < s.size() && (std::isalnum((unsigned char)s[p]) || s[p] == '_' || s[p] == '-' ||
                            s[p] == '.' || s[p] == ':'))
      ++p;
    if (b == p) throw std::runtime_error("XML name expected");
    return s.substr(b, p - b);
  }
  static std::string decode(std::string const& t) {
    std::string o;
    for (size_t i = 0; i < t.size(); ++i) {
      if (t[i] != '&') { o += t[i]; continue; }
      size_t e = t.find(';', i);
      std::string ent = e == std::string::npos ? "" : t.substr(i + 1, e - i - 1);
      if (ent == "lt") o += '<';
      else if (ent == "gt") o += '>';
      else if (ent == "amp") o += '&';
      else if (ent == "quot") o += '"';
      else if (ent == "apos") o += '\'';
      else { o += t[i]; continue; }
      i = e;
    }
    return o;
  }
  void ws() { while (p < s.size() && std::isspace((unsigned char)s[p])) ++p; }
  DOMElement* element() {
    ++p;   // '<'
    DOMElement* e = new DOMElement();
    e->m_name = u16(name());
    for (;;) {
      ws();
      if (starts("/>")) { p += 2; return e; }
      if (starts(">")) { ++p; break; }
      std::string a = name();
      ws();
      if (!starts("=")) throw std::runtime_error("'=' expected");
      ++p;
      ws();
      char q = s[p++];
      size_t end = s.find(q, p);
      e->setAttribute(u16(a).c_str(), u16(decode(s.substr(p, end - p))).c_str());
      p = end + 1;
    }
    for (;;) {
      if (p >= s.size()) throw std::runtime_error("unterminated element");
      if (starts("</")) {
        p += 2;
        name();
        ws();
        ++p;
        return e;
      }
      if (skipMisc()) continue;
      if (starts("<")) { e->appendChild(element()); continue; }
      size_t end = s.find('<', p);
      if (end == std::string::npos) end = s.size();
      DOMText* t = new DOMText();
      t->m_name = u"#text";
      t->m_value = u16(decode(s.substr(p, end - p)));
      e->appendChild(t);
      p = end;
    }
  }
};

}  // namespace

DOMDocument* DOMBuilder::parseURI(const char* path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    DOMException e;
    e.code = 1;
    e.msg = u"cannot open file";
    throw e;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  std::string text = ss.str();
  Parser P(text);
  DOMDocument* doc = new DOMDocument();
  for (;;) {
    P.ws();
    if (!P.skipMisc()) break;
  }
  doc->appendChild(P.element());
  return doc;
}

// --------------------------------------------------------------- writer --
static void writeXml(DOMNode const& n, std::string& out, int depth) {
  if (n.m_type == DOMNode::DOCUMENT_NODE) {
    out += "<?xml version=\"1.0\" encoding=\"UTF-8\" standalone=\"no\" ?>\n";
    for (DOMNode* c : n.m_children) writeXml(*c, out, depth);
    return;
  }
  if (n.m_type == DOMNode::TEXT_NODE) { out += u8(n.m_value); return; }
  out += std::string(2 * depth, ' ') + "<" + u8(n.m_name);
  for (DOMNode* a : n.m_attrs) out += " " + u8(a->m_name) + "=\"" + u8(a->m_value) + "\"";
  if (n.m_children.empty()) { out += "/>\n"; return; }
  bool textOnly = n.m_children.size() == 1 && n.m_children[0]->m_type == DOMNode::TEXT_NODE;
  out += ">";
  if (textOnly) {
    writeXml(*n.m_children[0], out, 0);
  } else {
    out += "\n";
    for (DOMNode* c : n.m_children) writeXml(*c, out, depth + 1);
    out += std::string(2 * depth, ' ');
  }
  out += "</" + u8(n.m_name) + ">\n";
}

bool DOMWriter::writeNode(XMLFormatTarget* target, DOMNode const& node) {
  LocalFileFormatTarget* f = dynamic_cast<LocalFileFormatTarget*>(target);
  if (!f) return false;
  writeXml(node, f->m_buffer, 0);
  return true;
}

void LocalFileFormatTarget::flush() {
  std::ofstream o(m_path, std::ios::binary);
  o << m_buffer;
}

DOMBuilder* DOMImplementation::createDOMBuilder(short, const XMLCh*) { return new DOMBuilder(); }
DOMDocument* DOMImplementation::createDocument(const XMLCh*, const XMLCh* qname, void*) {
  DOMDocument* d = new DOMDocument();
  d->appendChild(d->createElement(qname));
  return d;
}
DOMWriter* DOMImplementation::createDOMWriter() { return new DOMWriter(); }
DOMImplementation* DOMImplementationRegistry::getDOMImplementation(const XMLCh*) {
  static DOMImplementation impl;
  return &impl;
}
