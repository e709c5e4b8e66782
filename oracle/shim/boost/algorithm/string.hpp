// Test-infrastructure shim: the three Boost string algorithms the reference's
// readers call (trim, split with is_any_of, token_compress_on), written on top
// of the standard library so the reference sources compile without Boost.
// Only the oracle build (oracle/Makefile) puts this directory on the include path.
#pragma once
#include <cctype>
#include <string>
#include <vector>

namespace boost {
namespace algorithm {

enum token_compress_mode_type { token_compress_off, token_compress_on };

struct any_of_pred {
    std::string set;
    bool operator()(char c) const { return set.find(c) != std::string::npos; }
};

inline any_of_pred is_any_of(const std::string& s) { return any_of_pred{ s }; }

inline void trim(std::string& s)
{
    size_t b = 0, e = s.size();
    while (b < e && std::isspace(static_cast<unsigned char>(s[b]))) b++;
    while (e > b && std::isspace(static_cast<unsigned char>(s[e - 1]))) e--;
    s = s.substr(b, e - b);
}

// Split `in` at every character matched by `pred`.  With token_compress_on a
// run of adjacent separators counts as one; empty leading/trailing tokens are
// kept, as Boost does.
template <class Seq>
Seq& split(Seq& out, const std::string& in, any_of_pred pred,
    token_compress_mode_type mode = token_compress_off)
{
    out.clear();
    std::string cur;
    size_t i = 0;
    while (i < in.size()) {
        if (pred(in[i])) {
            out.push_back(cur);
            cur.clear();
            i++;
            if (mode == token_compress_on)
                while (i < in.size() && pred(in[i])) i++;
        } else {
            cur.push_back(in[i]);
            i++;
        }
    }
    out.push_back(cur);
    return out;
}

} // namespace algorithm
using algorithm::is_any_of;
using algorithm::split;
using algorithm::token_compress_on;
using algorithm::token_compress_off;
} // namespace boost
