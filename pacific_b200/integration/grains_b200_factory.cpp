// grains_b200_factory.cpp -- the "B200" branch of GrainsBuilderFactory::create
// (Base/src/GrainsBuilderFactory.cpp:16-40) for a Grains3D build that is
// linked, not patched.
//
// A Grains3D build that adds this library would add one line to the factory:
//     else if ( option == "B200" ) grains = new GrainsB200();
// The executable made by build_grains_b200.sh keeps every reference source
// unmodified instead: it is linked with --wrap on the factory's create(), so
// that the reference's own main() (GRAINS_V1/Main/src/main.cpp) reaches this
// function, which returns a GrainsB200 for Type="B200" and hands every other
// type to the reference's factory.  For B200 the factory's space-dimension
// context (set by create() from the root element's name) is set by running
// its Standard branch once on the same root.
#include <string>

#include "GrainsB200.hh"
#include "GrainsBuilderFactory.hh"
#include "ReaderXML.hh"

extern "C" {

Grains* __real__ZN20GrainsBuilderFactory6createEP10DOMElement(DOMElement* root);

Grains* __wrap__ZN20GrainsBuilderFactory6createEP10DOMElement(DOMElement* root) {
  if (ReaderXML::getNodeAttr_String(root, "Type") != "B200")
    return __real__ZN20GrainsBuilderFactory6createEP10DOMElement(root);
  XMLCh* name = XMLString::transcode("Type");
  XMLCh* standard = XMLString::transcode("Standard");
  XMLCh* b200 = XMLString::transcode("B200");
  root->setAttribute(name, standard);
  delete __real__ZN20GrainsBuilderFactory6createEP10DOMElement(root);
  root->setAttribute(name, b200);
  XMLString::release(&name);
  XMLString::release(&standard);
  XMLString::release(&b200);
  return new GrainsB200();
}

}  // extern "C"
