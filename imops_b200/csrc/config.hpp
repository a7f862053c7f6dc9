// config.hpp -- a small value tree and the two config grammars the reference
// accepts in parse_config (pichromatic-pipeline/src/config.rs:13-34): TOML
// (tried first) and JSON.  Only what pipeline configs use is supported:
// [[tables]] arrays, key = value, strings, integers, floats, booleans,
// arrays, inline tables, comments.
#pragma once

#include <map>
#include <memory>
#include <string>
#include <vector>

namespace imops {
namespace cfg {

struct Value {
    enum Kind { NUL, BOOL, INT, FLOAT, STRING, ARRAY, TABLE } kind = NUL;
    bool b = false;
    long long i = 0;
    double f = 0.0;
    std::string s;
    std::vector<Value> a;
    std::vector<std::pair<std::string, Value>> t;  // insertion-ordered table

    const Value* get(const std::string& key) const {
        for (auto& kv : t)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
    Value* get_mut(const std::string& key) {
        for (auto& kv : t)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
    bool is_number() const { return kind == INT || kind == FLOAT; }
    double number() const { return kind == INT ? (double)i : f; }
};

// Both return true on success; `err` receives a message otherwise.
bool parse_toml(const std::string& text, Value* out, std::string* err);
bool parse_json(const std::string& text, Value* out, std::string* err);

// JSON serialisation (for schema / metadata strings).
std::string to_json(const Value& v);

}  // namespace cfg
}  // namespace imops
