// Minimal JSON reader for EFEM configuration files (objects, arrays, strings,
// numbers, booleans, null).  Parses the whole document into a tree; no
// streaming, no unicode escapes beyond \uXXXX -> '?'.
#pragma once
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace efem {

struct Json {
    enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;  // insertion order kept

    bool is_number() const { return kind == NUM; }
    bool is_string() const { return kind == STR; }
    bool is_array() const { return kind == ARR; }
    bool is_object() const { return kind == OBJ; }
    bool is_bool() const { return kind == BOOL; }

    const Json* find(const std::string& key) const
    {
        if (kind != OBJ) return nullptr;
        for (auto& kv : obj)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
    double number_or(const std::string& key, double dflt) const
    {
        const Json* j = find(key);
        return (j && j->is_number()) ? j->num : dflt;
    }
};

class JsonParser {
public:
    explicit JsonParser(const std::string& s) : s_(s) { }
    Json parse()
    {
        Json j = value();
        ws();
        if (p_ != s_.size()) fail("trailing characters");
        return j;
    }

private:
    const std::string& s_;
    size_t p_ = 0;

    [[noreturn]] void fail(const char* what)
    {
        throw std::runtime_error(std::string("json: ") + what + " at offset " + std::to_string(p_));
    }
    void ws()
    {
        while (p_ < s_.size() && (s_[p_] == ' ' || s_[p_] == '\t' || s_[p_] == '\n' || s_[p_] == '\r')) p_++;
    }
    bool eat(const char* lit)
    {
        size_t n = std::char_traits<char>::length(lit);
        if (s_.compare(p_, n, lit) == 0) {
            p_ += n;
            return true;
        }
        return false;
    }
    Json value()
    {
        ws();
        if (p_ >= s_.size()) fail("unexpected end");
        char c = s_[p_];
        Json j;
        if (c == '{') {
            j.kind = Json::OBJ;
            p_++;
            ws();
            if (p_ < s_.size() && s_[p_] == '}') {
                p_++;
                return j;
            }
            for (;;) {
                ws();
                if (p_ >= s_.size() || s_[p_] != '"') fail("expected key");
                std::string k = string();
                ws();
                if (p_ >= s_.size() || s_[p_] != ':') fail("expected ':'");
                p_++;
                j.obj.emplace_back(k, value());
                ws();
                if (p_ < s_.size() && s_[p_] == ',') {
                    p_++;
                    continue;
                }
                if (p_ < s_.size() && s_[p_] == '}') {
                    p_++;
                    return j;
                }
                fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            j.kind = Json::ARR;
            p_++;
            ws();
            if (p_ < s_.size() && s_[p_] == ']') {
                p_++;
                return j;
            }
            for (;;) {
                j.arr.push_back(value());
                ws();
                if (p_ < s_.size() && s_[p_] == ',') {
                    p_++;
                    continue;
                }
                if (p_ < s_.size() && s_[p_] == ']') {
                    p_++;
                    return j;
                }
                fail("expected ',' or ']'");
            }
        }
        if (c == '"') {
            j.kind = Json::STR;
            j.str = string();
            return j;
        }
        if (eat("true")) {
            j.kind = Json::BOOL;
            j.b = true;
            return j;
        }
        if (eat("false")) {
            j.kind = Json::BOOL;
            return j;
        }
        if (eat("null")) return j;
        // number
        const char* b = s_.c_str() + p_;
        char* e = nullptr;
        double v = std::strtod(b, &e);
        if (e == b) fail("bad token");
        p_ += e - b;
        j.kind = Json::NUM;
        j.num = v;
        return j;
    }
    std::string string()
    {
        std::string out;
        p_++;  // opening quote
        while (p_ < s_.size() && s_[p_] != '"') {
            char c = s_[p_++];
            if (c == '\\') {
                if (p_ >= s_.size()) fail("bad escape");
                char e = s_[p_++];
                switch (e) {
                case 'n': out.push_back('\n'); break;
                case 't': out.push_back('\t'); break;
                case 'r': out.push_back('\r'); break;
                case 'b': out.push_back('\b'); break;
                case 'f': out.push_back('\f'); break;
                case 'u': p_ += 4; out.push_back('?'); break;
                default: out.push_back(e);
                }
            } else {
                out.push_back(c);
            }
        }
        if (p_ >= s_.size()) fail("unterminated string");
        p_++;
        return out;
    }
};

}  // namespace efem
