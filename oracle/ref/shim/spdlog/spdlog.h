// Test-infrastructure shim: a stand-in for the spdlog logging library so the
// reference's own sources (UQCreator code/src) compile in the oracle harness.
// spdlog is a third-party dependency of the reference (empty submodule
// code/ext/spdlog, commit unknown); only the calls made by the hot-path files
// are provided: spdlog::get(name)->info/error/warn/flush(fmt, args...).
//
// Behaviour chosen for the harness:
//   * info/warn: messages are dropped, except that the harness can capture the
//     "moments"/"duals" export lines (MomentSolver::Export, momentsolver.cpp:565-588).
//   * error: throws uqc_ref_error. The reference calls exit(EXIT_FAILURE) right
//     after logging an error (closure.cpp:180-192, vectorspace.cpp:166-170); the
//     harness turns that into a catchable error so the calling process survives.
#pragma once
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

struct uqc_ref_error : public std::runtime_error {
    explicit uqc_ref_error( const std::string& m ) : std::runtime_error( m ) {}
};

namespace spdlog {

namespace detail {
inline void fmt_append( std::ostringstream& os, const char* f ) { os << f; }
template <class A, class... R> void fmt_append( std::ostringstream& os, const char* f, const A& a, const R&... r ) {
    // Replace the first "{...}" placeholder by the argument; good enough for messages.
    while( *f ) {
        if( *f == '{' ) {
            const char* e = f;
            while( *e && *e != '}' ) ++e;
            os << a;
            fmt_append( os, *e ? e + 1 : e, r... );
            return;
        }
        os << *f++;
    }
}
}    // namespace detail

class logger
{
  public:
    explicit logger( std::string name ) : _name( std::move( name ) ) {}
    template <class... A> void info( const char* f, const A&... a ) { capture( f, a... ); }
    template <class... A> void info( const std::string& f, const A&... a ) { capture( f.c_str(), a... ); }
    template <class... A> void warn( const char*, const A&... ) {}
    template <class... A> void error( const char* f, const A&... a ) {
        std::ostringstream os;
        detail::fmt_append( os, f, a... );
        throw uqc_ref_error( os.str() );
    }
    template <class... A> void error( const std::string& f, const A&... a ) { error( f.c_str(), a... ); }
    void flush() {}

    // Harness-side capture of exported lines (used for the "moments"/"duals" loggers).
    bool capture_enabled = false;
    std::vector<std::string> lines;

  private:
    template <class... A> void capture( const char* f, const A&... a ) {
        if( !capture_enabled ) return;
        std::ostringstream os;
        detail::fmt_append( os, f, a... );
        lines.push_back( os.str() );
    }
    std::string _name;
};

inline std::shared_ptr<logger> get( const std::string& name ) {
    static std::map<std::string, std::shared_ptr<logger>> reg;
    auto& p = reg[name];
    if( !p ) p = std::make_shared<logger>( name );
    return p;
}

}    // namespace spdlog
