// grains_dom_shim.hpp -- minimal DOM with the Xerces-C 2.x names that the
// Grains3D XML layer (GRAINS_V1/Grains/XML/src/ReaderXML.cpp, WriterXML.cpp)
// uses, so the reference can be compiled unmodified as the serial oracle.
// TEST INFRASTRUCTURE ONLY.
//
// Behaviour kept from Xerces where the reference depends on it: text nodes
// (whitespace included) are children of their element; getChildNodes()
// returns a live list; getElementsByTagName() searches the subtree in
// document order; DOCTYPE declarations and comments are skipped; schema /
// DTD validation is not performed (the reference turns it off).
#ifndef GRAINS_DOM_SHIM_HPP
#define GRAINS_DOM_SHIM_HPP

// The Xerces-C headers bring in the C limits and stdlib declarations, which
// some reference sources rely on (INT_MAX, random()).
#include <climits>
#include <cstddef>
#include <cstdlib>
#include <string>
#include <vector>

#define XERCES_CPP_NAMESPACE_USE
#define XERCES_STD_QUALIFIER std::

typedef char16_t XMLCh;
typedef std::size_t XMLSize_t;

const XMLCh chNull = 0;
const XMLCh chLatin_L = u'L';
const XMLCh chLatin_S = u'S';

class DOMNodeList;
class DOMNamedNodeMap;
class DOMDocument;

class DOMNode {
 public:
  enum NodeType { ELEMENT_NODE = 1, ATTRIBUTE_NODE = 2, TEXT_NODE = 3, DOCUMENT_NODE = 9 };
  explicit DOMNode(short type);
  virtual ~DOMNode();
  const XMLCh* getNodeName() const { return m_name.c_str(); }
  const XMLCh* getNodeValue() const { return m_type == ELEMENT_NODE ? nullptr : m_value.c_str(); }
  short getNodeType() const { return m_type; }
  DOMNode* getFirstChild() const { return m_children.empty() ? nullptr : m_children.front(); }
  DOMNodeList* getChildNodes() const;
  DOMNamedNodeMap* getAttributes() const;
  DOMNode* cloneNode(bool deep) const;
  DOMNode* removeChild(DOMNode* old);
  DOMNode* appendChild(DOMNode* n);

  std::u16string m_name, m_value;
  short m_type;
  std::vector<DOMNode*> m_children;
  std::vector<DOMNode*> m_attrs;      // ATTRIBUTE_NODEs (name, value)
  DOMNode* m_parent = nullptr;
  mutable DOMNodeList* m_childList = nullptr;
  mutable DOMNamedNodeMap* m_attrMap = nullptr;
};

class DOMElement : public DOMNode {
 public:
  DOMElement() : DOMNode(ELEMENT_NODE) {}
  DOMNodeList* getElementsByTagName(const XMLCh* name) const;
  void setAttribute(const XMLCh* name, const XMLCh* value);
};

class DOMText : public DOMNode {
 public:
  DOMText() : DOMNode(TEXT_NODE) {}
};

class DOMNodeList {
 public:
  // live view of a node's children, or an owned snapshot
  explicit DOMNodeList(std::vector<DOMNode*> const* live) : m_live(live) {}
  explicit DOMNodeList(std::vector<DOMNode*> items) : m_live(nullptr), m_items(std::move(items)) {}
  DOMNode* item(XMLSize_t i) const {
    std::vector<DOMNode*> const& v = m_live ? *m_live : m_items;
    return i < v.size() ? v[i] : nullptr;
  }
  XMLSize_t getLength() const { return m_live ? m_live->size() : m_items.size(); }

 private:
  std::vector<DOMNode*> const* m_live;
  std::vector<DOMNode*> m_items;
};

class DOMNamedNodeMap {
 public:
  explicit DOMNamedNodeMap(std::vector<DOMNode*> const* attrs) : m_attrs(attrs) {}
  DOMNode* getNamedItem(const XMLCh* name) const;
  XMLSize_t getLength() const { return m_attrs->size(); }
  DOMNode* item(XMLSize_t i) const { return i < m_attrs->size() ? (*m_attrs)[i] : nullptr; }

 private:
  std::vector<DOMNode*> const* m_attrs;
};

class DOMDocument : public DOMNode {
 public:
  DOMDocument() : DOMNode(DOCUMENT_NODE) {}
  DOMElement* getDocumentElement() const;
  DOMElement* createElement(const XMLCh* name);
  DOMText* createTextNode(const XMLCh* data);
};

class DOMException {
 public:
  short code = 0;
  const XMLCh* msg = u"";
};

class IOException {};

class XMLFormatTarget {
 public:
  virtual ~XMLFormatTarget() {}
  virtual void flush() {}
};

class LocalFileFormatTarget : public XMLFormatTarget {
 public:
  explicit LocalFileFormatTarget(const char* path) : m_path(path) {}
  void flush() override;
  std::string m_path;
  std::string m_buffer;
};

class DOMBuilder {
 public:
  void setFeature(const XMLCh*, bool) {}
  DOMDocument* parseURI(const char* path);
};

class DOMWriter {
 public:
  void setFeature(const XMLCh*, bool) {}
  bool writeNode(XMLFormatTarget* target, DOMNode const& node);
};

class DOMImplementationLS {
 public:
  enum { MODE_SYNCHRONOUS = 1, MODE_ASYNCHRONOUS = 2 };
};

class DOMImplementation : public DOMImplementationLS {
 public:
  DOMBuilder* createDOMBuilder(short mode, const XMLCh* schemaType);
  DOMDocument* createDocument(const XMLCh* nsuri, const XMLCh* qname, void* doctype);
  DOMWriter* createDOMWriter();
};

class DOMImplementationRegistry {
 public:
  static DOMImplementation* getDOMImplementation(const XMLCh* features);
};

class AbstractDOMParser {};

class XMLString {
 public:
  static XMLCh* transcode(const char* s);
  static char* transcode(const XMLCh* s);
  static void release(char** p);
  static void release(XMLCh** p);
};

class XMLPlatformUtils {
 public:
  static void Initialize() {}
  static void Terminate() {}
};

namespace XMLUni {
extern const XMLCh fgDOMNamespaces[];
extern const XMLCh fgXercesSchema[];
extern const XMLCh fgXercesSchemaFullChecking[];
extern const XMLCh fgDOMDatatypeNormalization[];
extern const XMLCh fgDOMWRTFormatPrettyPrint[];
extern const XMLCh fgDOMValidation[];
}  // namespace XMLUni

#endif
