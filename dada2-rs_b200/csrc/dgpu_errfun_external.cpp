// The external-command error-model fit of learn-errors (external_errfun,
// src/error_models.rs:650-780): the transition matrix goes to a TSV file, a
// user command fits it and writes the error matrix to a second TSV file,
// which is parsed and checked. Host code, POSIX.
//
// The files use R's read.table(row.names = 1, header = TRUE) layout: a header
// of a tab and the quality scores 0..nq-1, then 16 rows, each a label (A2A,
// A2C, ..., T2T) and nq tab-separated values. The command is split on
// whitespace (no shell) and gets the two paths as its last arguments; its
// standard error is kept for the message when it fails. The messages and the
// checks (field counts, at most 16 data rows, numbers as Rust's f64 parser
// reads them, every value finite and in [0, 1]) follow the reference.
#include <dirent.h>
#include <fcntl.h>
#include <signal.h>
#include <spawn.h>
#include <sys/stat.h>
#include <sys/wait.h>
#include <unistd.h>

#include <atomic>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "dada2_b200.h"

extern char** environ;

namespace dgpu {
namespace {

const char* const kRowLabels[16] = {"A2A", "A2C", "A2G", "A2T", "C2A", "C2C", "C2G", "C2T",
                                    "G2A", "G2C", "G2G", "G2T", "T2A", "T2C", "T2G", "T2T"};

// An OS error as Rust's io::Error prints it.
std::string os_error(int e) { return std::string(std::strerror(e)) + " (os error " + std::to_string(e) + ")"; }

// The temporary folder, removed with what the command left in it.
struct TempFolder {
  std::string path;
  ~TempFolder() {
    if (path.empty()) return;
    std::vector<std::string> names;
    if (DIR* d = opendir(path.c_str())) {
      while (dirent* e = readdir(d))
        if (std::strcmp(e->d_name, ".") != 0 && std::strcmp(e->d_name, "..") != 0) names.push_back(e->d_name);
      closedir(d);
    }
    for (const std::string& n : names) std::remove((path + "/" + n).c_str());
    rmdir(path.c_str());
  }
};

// Rust's `f64` Display: the shortest digits that read back to the value, in
// positional notation (no exponent).
std::string rust_display(double v) {
  if (std::isnan(v)) return "NaN";
  if (std::isinf(v)) return v < 0 ? "-inf" : "inf";
  char buf[64];
  int prec = 1;
  for (; prec <= 17; ++prec) {
    std::snprintf(buf, sizeof buf, "%.*e", prec - 1, v);
    if (std::strtod(buf, nullptr) == v) break;
  }
  // buf = [-]d.ddde[+-]xx
  std::string s(buf);
  const bool neg = s[0] == '-';
  if (neg) s.erase(0, 1);
  const size_t epos = s.find('e');
  const int ex = std::atoi(s.c_str() + epos + 1);
  std::string digits;
  for (size_t i = 0; i < epos; ++i)
    if (s[i] != '.') digits += s[i];
  while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
  std::string out;
  const int point = ex + 1;  // digits before the decimal point
  if (point <= 0) {
    out = "0." + std::string(size_t(-point), '0') + digits;
  } else if (size_t(point) >= digits.size()) {
    out = digits + std::string(size_t(point) - digits.size(), '0');
  } else {
    out = digits.substr(0, size_t(point)) + "." + digits.substr(size_t(point));
  }
  if (v == 0.0) out = "0";
  return (neg ? "-" : "") + out;
}

// Rust's `{:?}` of a string (the common escapes).
std::string rust_debug(const std::string& s) {
  std::string o = "\"";
  for (unsigned char c : s) {
    if (c == '"') o += "\\\"";
    else if (c == '\\') o += "\\\\";
    else if (c == '\t') o += "\\t";
    else if (c == '\n') o += "\\n";
    else if (c == '\r') o += "\\r";
    else if (c < 0x20 || c == 0x7f) {
      char b[16];
      std::snprintf(b, sizeof b, "\\u{%x}", c);
      o += b;
    } else {
      o += char(c);
    }
  }
  return o + "\"";
}

// A number as Rust's `str::parse::<f64>` accepts it: an optional sign, then
// inf / infinity / nan (any case) or decimal digits with an optional point
// and exponent; nothing around it. On failure *why is Rust's message.
bool rust_parse_f64(const std::string& s, double* out, std::string* why) {
  if (s.empty()) {
    *why = "cannot parse float from empty string";
    return false;
  }
  size_t i = 0;
  if (s[i] == '+' || s[i] == '-') ++i;
  std::string rest = s.substr(i);
  std::string low;
  for (char c : rest) low += char(std::tolower(static_cast<unsigned char>(c)));
  bool ok = false;
  if (low == "inf" || low == "infinity" || low == "nan") {
    ok = true;
  } else {
    size_t k = 0, mant = 0;
    while (k < rest.size() && std::isdigit(static_cast<unsigned char>(rest[k]))) ++k, ++mant;
    if (k < rest.size() && rest[k] == '.') {
      ++k;
      while (k < rest.size() && std::isdigit(static_cast<unsigned char>(rest[k]))) ++k, ++mant;
    }
    ok = mant > 0;
    if (ok && k < rest.size() && (rest[k] == 'e' || rest[k] == 'E')) {
      ++k;
      if (k < rest.size() && (rest[k] == '+' || rest[k] == '-')) ++k;
      size_t ed = 0;
      while (k < rest.size() && std::isdigit(static_cast<unsigned char>(rest[k]))) ++k, ++ed;
      ok = ed > 0;
    }
    ok = ok && k == rest.size();
  }
  if (!ok) {
    *why = "invalid float literal";
    return false;
  }
  *out = std::strtod(s.c_str(), nullptr);
  return true;
}

std::vector<std::string> split(const std::string& s, char sep) {
  std::vector<std::string> v;
  size_t a = 0;
  for (;;) {
    const size_t b = s.find(sep, a);
    v.push_back(s.substr(a, b == std::string::npos ? std::string::npos : b - a));
    if (b == std::string::npos) break;
    a = b + 1;
  }
  return v;
}

// parse_err_tsv: the 16 x nq matrix of the command's output, or *msg.
bool parse_err_tsv(const std::string& text, int nq, double* err, std::string* msg) {
  // str::lines: split on '\n', each line without a trailing '\r'
  std::vector<std::string> lines = split(text, '\n');
  if (!lines.empty() && lines.back().empty()) lines.pop_back();
  for (std::string& l : lines)
    if (!l.empty() && l.back() == '\r') l.pop_back();
  if (lines.empty()) {
    *msg = "external_errfun: err TSV is empty";
    return false;
  }
  const size_t want = size_t(nq) + 1;
  const size_t hcols = split(lines[0], '\t').size();
  if (hcols != want) {
    *msg = "external_errfun: err TSV header has " + std::to_string(hcols) + " fields, expected " +
           std::to_string(want) + " (1 row-name + " + std::to_string(nq) + " quality scores)";
    return false;
  }
  int row = 0;
  for (size_t li = 1; li < lines.size(); ++li) {
    const std::string& line = lines[li];
    if (line.empty()) continue;
    if (row >= 16) {
      *msg = "external_errfun: err TSV has more than 16 data rows";
      return false;
    }
    const std::vector<std::string> cols = split(line, '\t');
    if (cols.size() != want) {
      *msg = "external_errfun: err TSV row " + std::to_string(row + 1) + " has " + std::to_string(cols.size()) +
             " fields, expected " + std::to_string(want);
      return false;
    }
    for (int q = 0; q < nq; ++q) {
      const std::string& cell = cols[size_t(q) + 1];
      double v = 0.0;
      std::string why;
      if (!rust_parse_f64(cell, &v, &why)) {
        *msg = "external_errfun: err TSV row " + std::to_string(row + 1) + " column " + std::to_string(q) + " (" +
               rust_debug(cell) + "): " + why;
        return false;
      }
      if (!std::isfinite(v) || !(v >= 0.0 && v <= 1.0)) {
        *msg = std::string("external_errfun: err[") + kRowLabels[row] + "][" + std::to_string(q) + "] = " +
               rust_display(v) + " is not a valid probability in [0, 1]";
        return false;
      }
      err[size_t(row) * nq + q] = v;
    }
    ++row;
  }
  if (row != 16) {
    *msg = "external_errfun: err TSV has " + std::to_string(row) + " data rows, expected 16";
    return false;
  }
  return true;
}

// An exit status as Rust's ExitStatus prints it on Unix.
std::string exit_text(int status) {
  if (WIFEXITED(status)) return "exit status: " + std::to_string(WEXITSTATUS(status));
  if (WIFSIGNALED(status)) {
    const int sg = WTERMSIG(status);
    const char* name = sigabbrev_np(sg);
    std::string t = "signal: " + std::to_string(sg);
    if (name) t += std::string(" (SIG") + name + ")";
    if (WCOREDUMP(status)) t += " (core dumped)";
    return t;
  }
  return "unknown status";
}

std::atomic<uint64_t> g_folder_seq{0};

}  // namespace

// external_errfun (src/error_models.rs:650-705).
int external_errfun_fit(const char* cmd_c, const uint32_t* trans, int nq, double* err, std::string* msg) {
  const std::string cmd = cmd_c ? cmd_c : "";
  std::vector<std::string> argv;
  {
    size_t i = 0;
    while (i < cmd.size()) {
      while (i < cmd.size() && std::isspace(static_cast<unsigned char>(cmd[i]))) ++i;
      size_t j = i;
      while (j < cmd.size() && !std::isspace(static_cast<unsigned char>(cmd[j]))) ++j;
      if (j > i) argv.push_back(cmd.substr(i, j - i));
      i = j;
    }
  }
  if (argv.empty()) {
    *msg = "external_errfun: --errfun-cmd is empty";
    return DGPU_E_INVALID;
  }
  TempFolder tmp;
  {
    // a folder this call creates itself (an existing one, which another user
    // could have planted, is never written into)
    const char* t = std::getenv("TMPDIR");
    const std::string base = (t && *t) ? t : "/tmp";
    int e = EEXIST;
    for (int tries = 0; tries < 100 && e == EEXIST; ++tries) {
      const std::string path = base + "/dada2-rs-errfun-" + std::to_string(getpid()) + "-" +
                               std::to_string(g_folder_seq.fetch_add(1));
      if (mkdir(path.c_str(), 0700) == 0) {
        tmp.path = path;
        e = 0;
      } else {
        e = errno;
      }
    }
    if (e != 0) {
      *msg = "external_errfun: failed to create temp dir: " + os_error(e);
      return DGPU_E_INVALID;
    }
  }
  const std::string trans_path = tmp.path + "/trans.tsv", err_path = tmp.path + "/err.tsv";
  {
    std::string body;
    for (int q = 0; q < nq; ++q) body += "\t" + std::to_string(q);
    body += "\n";
    for (int r = 0; r < 16; ++r) {
      body += kRowLabels[r];
      for (int q = 0; q < nq; ++q) body += "\t" + std::to_string(trans[size_t(r) * nq + q]);
      body += "\n";
    }
    FILE* f = std::fopen(trans_path.c_str(), "wb");
    const bool ok = f && std::fwrite(body.data(), 1, body.size(), f) == body.size();
    const int e = errno;
    if (f && std::fclose(f) != 0 && ok) {
      *msg = "external_errfun: write " + trans_path + ": " + os_error(errno);
      return DGPU_E_INVALID;
    }
    if (!ok) {
      *msg = "external_errfun: write " + trans_path + ": " + os_error(e);
      return DGPU_E_INVALID;
    }
  }
  // the command: no shell; standard output discarded, standard error kept
  std::vector<std::string> args = argv;
  args.push_back(trans_path);
  args.push_back(err_path);
  std::vector<char*> av;
  for (std::string& a : args) av.push_back(&a[0]);
  av.push_back(nullptr);
  int pipefd[2];
  if (pipe(pipefd) != 0) {
    *msg = "external_errfun: failed to spawn '" + cmd + "': " + os_error(errno);
    return DGPU_E_INVALID;
  }
  posix_spawn_file_actions_t fa;
  posix_spawn_file_actions_init(&fa);
  posix_spawn_file_actions_addopen(&fa, 1, "/dev/null", O_WRONLY, 0);
  posix_spawn_file_actions_adddup2(&fa, pipefd[1], 2);
  posix_spawn_file_actions_addclose(&fa, pipefd[0]);
  posix_spawn_file_actions_addclose(&fa, pipefd[1]);
  pid_t pid = 0;
  const int sp = posix_spawnp(&pid, av[0], &fa, nullptr, av.data(), environ);
  posix_spawn_file_actions_destroy(&fa);
  close(pipefd[1]);
  if (sp != 0) {
    close(pipefd[0]);
    *msg = "external_errfun: failed to spawn '" + cmd + "': " + os_error(sp);
    return DGPU_E_INVALID;
  }
  std::string errtext;
  char buf[4096];
  for (;;) {
    const ssize_t n = read(pipefd[0], buf, sizeof buf);
    if (n > 0) errtext.append(buf, size_t(n));
    else if (n == 0 || errno != EINTR) break;
  }
  close(pipefd[0]);
  int status = 0;
  while (waitpid(pid, &status, 0) < 0 && errno == EINTR) {
  }
  if (!(WIFEXITED(status) && WEXITSTATUS(status) == 0)) {
    while (!errtext.empty() && std::isspace(static_cast<unsigned char>(errtext.back()))) errtext.pop_back();
    *msg = "external_errfun: command '" + cmd + "' exited with " + exit_text(status) + "\n--- stderr ---\n" + errtext;
    return DGPU_E_INVALID;
  }
  std::string text;
  {
    FILE* f = std::fopen(err_path.c_str(), "rb");
    if (!f) {
      *msg = "external_errfun: read " + err_path + ": " + os_error(errno);
      return DGPU_E_INVALID;
    }
    size_t n;
    while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
    std::fclose(f);
  }
  return parse_err_tsv(text, nq, err, msg) ? 0 : DGPU_E_INVALID;
}

}  // namespace dgpu
