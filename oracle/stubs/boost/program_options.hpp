// Minimal stand-in for the part of boost::program_options that the hpHawkes
// benchmark CLI uses (src/benchmark.cpp:29-57): options_description with
// add_options(), value<int>()->default_value(), parse_command_line, store,
// notify, variables_map::count / operator[] / as<T>().  Boost is not installed
// in this image; this header lets benchmark.cpp compile unmodified so that the
// reference's own CLI can drive both the reference CPU engine and the CUDA
// engine through hph::factory.
//
// Supported syntax: "--name value", "--name=value" and bare "--flag".
// Unknown options throw std::runtime_error, which benchmark.cpp catches and
// reports by printing the description.
#ifndef HAWKES_ORACLE_PROGRAM_OPTIONS_STUB_HPP
#define HAWKES_ORACLE_PROGRAM_OPTIONS_STUB_HPP

#include <map>
#include <memory>
#include <ostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace boost {
namespace program_options {

class value_semantic {
public:
    virtual ~value_semantic() = default;
    virtual bool has_default() const = 0;
    virtual std::string default_text() const = 0;
};

template <typename T>
class typed_value : public value_semantic {
public:
    typed_value* default_value(const T& v) {
        def = v;
        hasDef = true;
        return this;
    }
    bool has_default() const override { return hasDef; }
    std::string default_text() const override {
        std::ostringstream s;
        s << def;
        return s.str();
    }
    T def{};
    bool hasDef = false;
};

template <typename T>
typed_value<T>* value() {
    return new typed_value<T>();
}

struct option {
    std::string name;
    std::string help;
    std::shared_ptr<value_semantic> semantic;  // null for a bare flag
};

class options_description;

class options_description_easy_init {
public:
    explicit options_description_easy_init(options_description* d) : owner(d) {}
    options_description_easy_init& operator()(const char* name, const char* help);
    options_description_easy_init& operator()(const char* name, value_semantic* s, const char* help);

private:
    options_description* owner;
};

class options_description {
public:
    explicit options_description(const std::string& caption = "") : caption(caption) {}
    options_description_easy_init add_options() { return options_description_easy_init(this); }
    const option* find(const std::string& name) const {
        for (auto& o : options)
            if (o.name == name) return &o;
        return nullptr;
    }
    std::string caption;
    std::vector<option> options;
};

inline options_description_easy_init& options_description_easy_init::operator()(const char* name,
                                                                                const char* help) {
    owner->options.push_back(option{name, help, nullptr});
    return *this;
}

inline options_description_easy_init& options_description_easy_init::operator()(const char* name,
                                                                                value_semantic* s,
                                                                                const char* help) {
    owner->options.push_back(option{name, help, std::shared_ptr<value_semantic>(s)});
    return *this;
}

inline std::ostream& operator<<(std::ostream& os, const options_description& d) {
    os << d.caption << ":\n";
    for (auto& o : d.options) {
        os << "  --" << o.name;
        if (o.semantic && o.semantic->has_default()) os << " arg (=" << o.semantic->default_text() << ")";
        os << "\t" << o.help << "\n";
    }
    return os;
}

class variable_value {
public:
    variable_value() = default;
    explicit variable_value(std::string t) : text(std::move(t)) {}
    template <typename T>
    T as() const {
        std::istringstream s(text);
        T v{};
        if (!(s >> v)) throw std::runtime_error("bad option value: " + text);
        return v;
    }
    std::string text;
};

class variables_map : public std::map<std::string, variable_value> {
public:
    const variable_value& operator[](const std::string& k) const {
        auto it = find(k);
        if (it == end()) throw std::runtime_error("option not set: " + k);
        return it->second;
    }
};

struct parsed_options {
    const options_description* desc = nullptr;
    std::map<std::string, std::string> given;
};

inline parsed_options parse_command_line(int argc, char** argv, const options_description& desc) {
    parsed_options p;
    p.desc = &desc;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if (a.rfind("--", 0) != 0) throw std::runtime_error("unexpected argument: " + a);
        a = a.substr(2);
        std::string val;
        bool hasVal = false;
        auto eq = a.find('=');
        if (eq != std::string::npos) {
            val = a.substr(eq + 1);
            a = a.substr(0, eq);
            hasVal = true;
        }
        const option* o = desc.find(a);
        if (!o) throw std::runtime_error("unknown option: " + a);
        if (o->semantic) {
            if (!hasVal) {
                if (i + 1 >= argc) throw std::runtime_error("missing value for: " + a);
                val = argv[++i];
            }
        } else if (hasVal) {
            throw std::runtime_error("flag takes no value: " + a);
        }
        p.given[a] = val;
    }
    return p;
}

inline void store(const parsed_options& p, variables_map& vm) {
    for (auto& o : p.desc->options) {
        auto it = p.given.find(o.name);
        if (it != p.given.end()) {
            vm.insert_or_assign(o.name, variable_value(it->second));
        } else if (o.semantic && o.semantic->has_default()) {
            vm.insert_or_assign(o.name, variable_value(o.semantic->default_text()));
        }
    }
}

inline void notify(variables_map&) {}

}  // namespace program_options
}  // namespace boost

#endif
