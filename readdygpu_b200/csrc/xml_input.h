// xml_input.h -- a small XML reader (elements, attributes, text, comments)
// for the ReaDDy input files.
#pragma once
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace rdxml {

struct Node {
    std::string name;
    std::map<std::string, std::string> attrs;
    std::string text;
    std::vector<std::unique_ptr<Node>> kids;
    const Node* child(const std::string& n) const;
    std::vector<const Node*> children(const std::string& n) const;
    std::string child_text(const std::string& n, const std::string& dflt = "") const;
};

// parses a document; returns the root element or null with an error message
std::unique_ptr<Node> parse(const std::string& src, std::string& err);
bool read_file(const std::string& path, std::string& out);
std::string trim(const std::string& s);

}  // namespace rdxml
