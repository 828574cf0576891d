// INFO-format reader (the subset of boost::property_tree's INFO grammar CAFFE case files use)
// and the Input / Vector3D helpers of the host layer.
#include "Input.h"
#include "Vector3D.h"

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace {

std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

// drop a ';' comment that is not inside a quoted string
std::string strip_comment(const std::string& s) {
    bool q = false;
    for (size_t i = 0; i < s.size(); ++i) {
        if (s[i] == '"') q = !q;
        else if (s[i] == ';' && !q) return s.substr(0, i);
    }
    return s;
}

std::string unquote(const std::string& s) {
    if (s.size() >= 2 && s.front() == '"' && s.back() == '"') return s.substr(1, s.size() - 2);
    return s;
}

}  // namespace

InfoTree InfoTree::parse(const std::string& text) {
    InfoTree root;
    std::vector<InfoTree*> stack{&root};
    InfoTree* last = nullptr;   // most recent key of the current level (a '{' opens it)
    std::istringstream in(text);
    std::string raw;
    int lineNo = 0;
    while (std::getline(in, raw)) {
        ++lineNo;
        std::string line = trim(strip_comment(raw));
        // strip a UTF-8 byte-order mark on the first line
        if (lineNo == 1 && line.size() >= 3 && (unsigned char)line[0] == 0xEF) line = trim(line.substr(3));
        while (!line.empty()) {
            if (line[0] == '{') {
                if (!last) Output::raiseException("InfoTree", "parse", "'{' without a key at line " + std::to_string(lineNo));
                stack.push_back(last);
                last = nullptr;
                line = trim(line.substr(1));
                continue;
            }
            if (line[0] == '}') {
                if (stack.size() <= 1) Output::raiseException("InfoTree", "parse", "unbalanced '}' at line " + std::to_string(lineNo));
                stack.pop_back();
                last = nullptr;
                line = trim(line.substr(1));
                continue;
            }
            // key [value] [{ | }]
            size_t ks = line.find_first_of(" \t{}");
            std::string key = line.substr(0, ks);
            std::string rest = ks == std::string::npos ? "" : line.substr(ks);
            std::string value;
            size_t brace = rest.find_first_of("{}");
            if (brace == std::string::npos) { value = trim(rest); rest.clear(); }
            else { value = trim(rest.substr(0, brace)); rest = rest.substr(brace); }
            InfoTree child;
            child.data = unquote(value);
            stack.back()->children.emplace_back(key, child);
            last = &stack.back()->children.back().second;
            line = trim(rest);
        }
    }
    if (stack.size() != 1) Output::raiseException("InfoTree", "parse", "unbalanced '{' at end of input");
    return root;
}

InfoTree InfoTree::readFile(const std::string& filename) {
    std::ifstream f(filename);
    if (!f) Output::raiseException("InfoTree", "readFile", "cannot open \"" + filename + "\"");
    std::stringstream ss;
    ss << f.rdbuf();
    return parse(ss.str());
}

const InfoTree* InfoTree::find(const std::string& path) const {
    const InfoTree* t = this;
    size_t pos = 0;
    while (pos <= path.size()) {
        size_t dot = path.find('.', pos);
        std::string key = path.substr(pos, dot == std::string::npos ? std::string::npos : dot - pos);
        const InfoTree* next = nullptr;
        for (const auto& c : t->children)
            if (c.first == key) { next = &c.second; break; }
        if (!next) return nullptr;
        t = next;
        if (dot == std::string::npos) break;
        pos = dot + 1;
    }
    return t;
}

std::string InfoTree::getString(const std::string& path) const {
    const InfoTree* t = find(path);
    if (!t) Output::raiseException("InfoTree", "get", "no key \"" + path + "\" in the input");
    return t->data;
}

template <>
std::string InfoTree::get<std::string>(const std::string& path) const { return getString(path); }

template <>
double InfoTree::get<double>(const std::string& path) const {
    std::string s = getString(path);
    char* end = nullptr;
    double v = std::strtod(s.c_str(), &end);
    if (end == s.c_str()) Output::raiseException("InfoTree", "get", "\"" + path + "\" is not a number: " + s);
    return v;
}

template <>
int InfoTree::get<int>(const std::string& path) const {
    std::string s = getString(path);
    char* end = nullptr;
    long v = std::strtol(s.c_str(), &end, 10);
    if (end == s.c_str()) Output::raiseException("InfoTree", "get", "\"" + path + "\" is not an integer: " + s);
    return (int)v;
}

Input::Input() : Input("case/case.info", "case/initialConditions.info") {}

Input::Input(const std::string& caseFilename, const std::string& initialConditionsFilename) {
    caseParameters = InfoTree::readFile(caseFilename);
    std::ifstream probe(initialConditionsFilename);
    if (probe) initialConditions = InfoTree::readFile(initialConditionsFilename);
}

Vector3D std::stov(const std::string& s) {
    std::string t;
    for (char ch : s)
        if (ch != '(' && ch != ')') t += (ch == ',' ? ' ' : ch);
    std::istringstream in(t);
    Vector3D v;
    if (!(in >> v.x >> v.y >> v.z)) Output::raiseException("Vector3D", "stov", "cannot read a vector from \"" + s + "\"");
    return v;
}
