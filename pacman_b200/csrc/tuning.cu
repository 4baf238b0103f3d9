// Launch parameters of the patch solvers, per GPU model.
//
// The tuner (python -m pacman_b200.tune) times whole transfers on the
// current GPU over a grid of these parameters and writes the fastest choice
// to tuning/<GPU name>.conf beside libpacman_b200.so, one "key = value" per
// line.  The library reads that file once per device (the first transfer on
// it); an environment variable of the same name overrides a value per call,
// and a missing file or key keeps the built-in default.
#include <dlfcn.h>

#include <cctype>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "plan.hpp"

namespace pacman_b200 {
namespace {

std::mutex g_tune_mu;
std::map<int, Tuning> g_tune;  // per device ordinal

std::string library_dir() {
  Dl_info info{};
  if (dladdr(reinterpret_cast<void *>(&tuning_for_current_device), &info) && info.dli_fname) {
    std::string p(info.dli_fname);
    const size_t s = p.rfind('/');
    return s == std::string::npos ? std::string(".") : p.substr(0, s);
  }
  return ".";
}

// "NVIDIA B200" -> "NVIDIA_B200".
std::string file_stem(const char *name) {
  std::string s;
  for (const char *c = name; *c; ++c)
    s += (std::isalnum(static_cast<unsigned char>(*c)) || *c == '-' || *c == '.') ? *c : '_';
  return s;
}

void parse(const std::string &path, Tuning &t) {
  std::ifstream f(path);
  if (!f) return;
  t.source = path;
  std::string line;
  while (std::getline(f, line)) {
    const size_t hash = line.find('#');
    if (hash != std::string::npos) line.resize(hash);
    const size_t eq = line.find('=');
    if (eq == std::string::npos) continue;
    auto trim = [](std::string x) {
      const size_t a = x.find_first_not_of(" \t\r");
      const size_t b = x.find_last_not_of(" \t\r");
      return a == std::string::npos ? std::string() : x.substr(a, b - a + 1);
    };
    const std::string key = trim(line.substr(0, eq)), val = trim(line.substr(eq + 1));
    const int v = std::atoi(val.c_str());
    if (key == "PACMAN_B200_BIG_N") t.big_n_chol = v;
    else if (key == "PACMAN_B200_INT8_FROM") t.int8_from = v;
    else if (key == "PACMAN_B200_GROUPS") t.groups = v;
    else if (key == "PACMAN_B200_BACK_STAGES") t.back_stages = v;
  }
}

}  // namespace

const Tuning &tuning_for_current_device() {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(g_tune_mu);
  auto it = g_tune.find(dev);
  if (it != g_tune.end()) return it->second;
  Tuning t;
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess) {
    t.sms = prop.multiProcessorCount;
    parse(library_dir() + "/tuning/" + file_stem(prop.name) + ".conf", t);
  }
  cudaGetLastError();
  return g_tune.emplace(dev, t).first->second;
}

int tuned_int(const char *env, int value) {
  const char *e = std::getenv(env);
  return e ? std::atoi(e) : value;
}

}  // namespace pacman_b200
