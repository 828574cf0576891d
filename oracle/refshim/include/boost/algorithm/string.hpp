// Stand-in for the boost string algorithms the reference's StructuredMesh.cpp uses to read a
// Tecplot header (test infrastructure): split on any of a set of characters, upper-casing.
#ifndef CAFFE_REFSHIM_ALGORITHM_STRING_HPP
#define CAFFE_REFSHIM_ALGORITHM_STRING_HPP

#include <cctype>
#include <string>
#include <vector>

namespace boost {
namespace algorithm {

enum token_compress_mode_type { token_compress_on, token_compress_off };

struct any_of_pred {
    std::string set;
    bool operator()(char c) const { return set.find(c) != std::string::npos; }
};
inline any_of_pred is_any_of(const std::string& s) { return any_of_pred{s}; }

inline std::vector<std::string>& split(std::vector<std::string>& out, const std::string& in, const any_of_pred& sep,
                                       token_compress_mode_type mode = token_compress_off) {
    out.clear();
    std::string cur;
    bool lastSep = false;
    for (char c : in) {
        if (sep(c)) {
            if (!(mode == token_compress_on && lastSep)) out.push_back(cur);
            cur.clear();
            lastSep = true;
        } else {
            cur.push_back(c);
            lastSep = false;
        }
    }
    out.push_back(cur);
    return out;
}
inline void to_upper(std::string& s) {
    for (char& c : s) c = (char)std::toupper((unsigned char)c);
}
inline std::string to_upper_copy(std::string s) {
    to_upper(s);
    return s;
}

}  // namespace algorithm
}  // namespace boost

#endif
