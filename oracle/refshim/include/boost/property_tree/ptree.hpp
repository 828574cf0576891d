// Stand-in for boost::property_tree::ptree as the reference's solver path uses it (test
// infrastructure): a tree of string-valued nodes addressed by dotted paths, with typed reads
// that parse the node's text by stream extraction and fail on a missing path or on text
// left over.
#ifndef CAFFE_REFSHIM_PTREE_HPP
#define CAFFE_REFSHIM_PTREE_HPP

#include <locale>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace boost {
namespace property_tree {

class ptree {
public:
    std::string data;
    std::vector<std::pair<std::string, ptree>> children;

    ptree* find(const std::string& path) {
        ptree* node = this;
        size_t pos = 0;
        while (node) {
            size_t dot = path.find('.', pos);
            std::string key = path.substr(pos, dot == std::string::npos ? std::string::npos : dot - pos);
            ptree* next = nullptr;
            for (auto& c : node->children)
                if (c.first == key) { next = &c.second; break; }
            node = next;
            if (dot == std::string::npos) break;
            pos = dot + 1;
        }
        return node;
    }
    const ptree* find(const std::string& path) const { return const_cast<ptree*>(this)->find(path); }

    ptree& put_child_path(const std::string& path) {
        ptree* node = this;
        size_t pos = 0;
        while (true) {
            size_t dot = path.find('.', pos);
            std::string key = path.substr(pos, dot == std::string::npos ? std::string::npos : dot - pos);
            ptree* next = nullptr;
            for (auto& c : node->children)
                if (c.first == key) { next = &c.second; break; }
            if (!next) {
                node->children.emplace_back(key, ptree());
                next = &node->children.back().second;
            }
            node = next;
            if (dot == std::string::npos) return *node;
            pos = dot + 1;
        }
    }

    template <class T>
    static bool convert(const std::string& s, T& out) {
        std::istringstream is(s);
        is.imbue(std::locale::classic());
        is >> out;
        if (is.fail()) return false;
        is >> std::ws;
        return is.eof();
    }

    template <class T>
    T get(const std::string& path) const {
        const ptree* n = find(path);
        if (!n) throw std::runtime_error("No such node (" + path + ")");
        T v;
        if (!convert(n->data, v)) throw std::runtime_error("conversion of data to type failed (" + path + ")");
        return v;
    }
    template <class T>
    T get(const std::string& path, const T& fallback) const {
        const ptree* n = find(path);
        T v;
        if (!n || !convert(n->data, v)) return fallback;
        return v;
    }
    template <class T>
    void put(const std::string& path, const T& value) {
        std::ostringstream os;
        os.imbue(std::locale::classic());
        os.precision(17);
        os << value;
        put_child_path(path).data = os.str();
    }
};

template <>
inline std::string ptree::get<std::string>(const std::string& path) const {
    const ptree* n = find(path);
    if (!n) throw std::runtime_error("No such node (" + path + ")");
    return n->data;
}
template <>
inline std::string ptree::get<std::string>(const std::string& path, const std::string& fallback) const {
    const ptree* n = find(path);
    return n ? n->data : fallback;
}

}  // namespace property_tree
}  // namespace boost

#endif
