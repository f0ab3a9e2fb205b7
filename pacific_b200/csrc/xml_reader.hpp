// xml_reader.hpp -- minimal, non-validating XML reader for Grains3D input.
//
// Grains3D reads its input through a Xerces DOM wrapper (GRAINS_V1/Grains/
// XML/src/ReaderXML.cpp); the accessors below mirror the ones the DEM step
// needs from it: getNode (first element child by name), getNodes (element
// children), getNodeAttr_Double/Int/String, hasNodeAttr, getNodeValue_*.
// DTD declarations, processing instructions and comments are skipped, as the
// reference parser is configured without schema validation.
#pragma once
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace gdem {

struct XmlNode {
  std::string name;
  std::map<std::string, std::string> attrs;
  std::string text;                                   // concatenated character data
  std::vector<std::unique_ptr<XmlNode>> children;     // element children only

  XmlNode const* child(std::string const& n) const {
    for (auto const& c : children)
      if (c->name == n) return c.get();
    return nullptr;
  }
  std::vector<XmlNode const*> childrenNamed(std::string const& n) const {
    std::vector<XmlNode const*> out;
    for (auto const& c : children)
      if (c->name == n) out.push_back(c.get());
    return out;
  }
  // Depth-first search, like DOMElement::getElementsByTagName(name)->item(0)
  XmlNode const* find(std::string const& n) const {
    for (auto const& c : children) {
      if (c->name == n) return c.get();
      if (auto f = c->find(n)) return f;
    }
    return nullptr;
  }
  bool has(std::string const& a) const { return attrs.count(a) != 0; }
  std::string attr(std::string const& a) const {
    auto it = attrs.find(a);
    if (it == attrs.end()) throw std::runtime_error("XML: <" + name + "> lacks attribute " + a);
    return it->second;
  }
  double attrD(std::string const& a) const { return std::stod(attr(a)); }
  int attrI(std::string const& a) const { return std::stoi(attr(a)); }
  double valueD() const { return std::stod(text); }
  std::string valueS() const;
};

std::unique_ptr<XmlNode> parseXmlFile(std::string const& path);
std::unique_ptr<XmlNode> parseXmlString(std::string const& text);

}  // namespace gdem
