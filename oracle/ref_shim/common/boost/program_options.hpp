// Minimal stand-in for boost::program_options (TEST INFRASTRUCTURE ONLY).
// zephyr parses two options with it (--threads, --config); the checker never
// passes command-line arguments, so parsing yields each option's default.
#pragma once
#include <map>
#include <memory>
#include <string>

namespace boost {
namespace program_options {

class value_semantic {
public:
    virtual ~value_semantic() = default;
    std::string def;
};

template <class T>
class typed_value : public value_semantic {
public:
    typed_value *default_value(const T &v) {
        def = v;
        return this;
    }
};

template <class T>
typed_value<T> *value() {
    return new typed_value<T>();
}

class options_description {
public:
    struct adder {
        options_description *d;
        adder &operator()(const char *name, value_semantic *v) {
            std::string key(name);
            auto comma = key.find(',');
            if (comma != std::string::npos) key = key.substr(0, comma);
            d->defaults[key] = v->def;
            d->owned.emplace_back(v);
            return *this;
        }
    };
    adder add_options() { return adder{this}; }
    std::map<std::string, std::string> defaults;
    std::vector<std::unique_ptr<value_semantic>> owned;
};

class variable_value {
public:
    std::string v;
    template <class T>
    const T &as() const {
        return v;
    }
};

class variables_map : public std::map<std::string, variable_value> {};

struct parsed_options {
    std::map<std::string, std::string> values;
};

class command_line_parser {
public:
    command_line_parser(int, char **) {}
    command_line_parser &options(const options_description &d) {
        parsed.values = d.defaults;
        return *this;
    }
    command_line_parser &allow_unregistered() { return *this; }
    parsed_options run() { return parsed; }

private:
    parsed_options parsed;
};

inline void store(const parsed_options &p, variables_map &vm) {
    for (auto &kv : p.values) vm[kv.first].v = kv.second;
}
inline void notify(variables_map &) {}

}  // namespace program_options
}  // namespace boost
