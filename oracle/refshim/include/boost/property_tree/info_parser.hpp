// Stand-in for boost::property_tree::read_info (test infrastructure): reads the INFO files the
// reference's cases use -- "key value" lines, "key" followed by a "{ ... }" block (the brace on
// the same or the next line), ';' comments and double-quoted values.
#ifndef CAFFE_REFSHIM_INFO_PARSER_HPP
#define CAFFE_REFSHIM_INFO_PARSER_HPP

#include <string>

#include "ptree.hpp"

namespace boost {
namespace property_tree {
namespace info_parser {
void read_info(const std::string& filename, ptree& pt);
}
using info_parser::read_info;
}  // namespace property_tree
}  // namespace boost

#endif
