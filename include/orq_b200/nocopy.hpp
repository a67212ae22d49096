// nocopy.hpp — ORQ's NoCopy wire, so a GPU party can sit among CPU parties.
//
// The reference's NoCopy communicator (core/communication/no_copy_communicator/
// no_copy_communicator.h:120-266) sends every vector as its raw little-endian
// bytes, with no header, over one TCP socket per pair of parties and worker
// thread; sizes are implied by the protocol. Sockets are set up by startmpc
// (backend/nocopy_communicator/startmpc/startmpc.h): with H hosts and T
// threads, host i connects to every host j > i on ports base + H*T*i + T*j + t
// and host j listens on the same ports. The environment names the roles:
// STARTMPC_EXEC_MODE (0 local, 1 remote with STARTMPC_HOST_LIST),
// STARTMPC_HOST_COUNT, STARTMPC_HOST_RANK, STARTMPC_BASE_PORT.
//
// This endpoint speaks that format for one worker thread (a CPU party run
// with `1 1 -1`, the configuration whose shares the GPU party reproduces).
#pragma once

#include <arpa/inet.h>
#include <netdb.h>
#include <netinet/in.h>
#include <sys/socket.h>
#include <unistd.h>

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace orq {
namespace nocopy {

struct WireError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

class Endpoint {
    int rank_ = 0, count_ = 0;
    std::vector<int> fd_;

    static int listen_accept(int port) {
        const int s = ::socket(AF_INET, SOCK_STREAM, 0);
        if (s < 0) throw WireError("socket failed");
        int one = 1;
        ::setsockopt(s, SOL_SOCKET, SO_REUSEADDR, &one, sizeof(one));
        sockaddr_in a{};
        a.sin_family = AF_INET;
        a.sin_addr.s_addr = INADDR_ANY;
        a.sin_port = htons((uint16_t)port);
        if (::bind(s, (sockaddr*)&a, sizeof(a)) != 0) {
            ::close(s);
            throw WireError("bind failed on port " + std::to_string(port));
        }
        if (::listen(s, 1) != 0) {
            ::close(s);
            throw WireError("listen failed on port " + std::to_string(port));
        }
        const int c = ::accept(s, nullptr, nullptr);
        ::close(s);
        if (c < 0) throw WireError("accept failed on port " + std::to_string(port));
        return c;
    }

    // the peer may start later: retry for up to `wait_s` seconds
    static int connect_to(const std::string& host, int port, int wait_s) {
        addrinfo hints{}, *res = nullptr;
        hints.ai_family = AF_INET;
        hints.ai_socktype = SOCK_STREAM;
        if (::getaddrinfo(host.c_str(), std::to_string(port).c_str(), &hints, &res) != 0)
            throw WireError("cannot resolve " + host);
        const auto until = std::chrono::steady_clock::now() + std::chrono::seconds(wait_s);
        for (;;) {
            const int s = ::socket(res->ai_family, res->ai_socktype, res->ai_protocol);
            if (s < 0) {
                ::freeaddrinfo(res);
                throw WireError("socket failed");
            }
            if (::connect(s, res->ai_addr, res->ai_addrlen) == 0) {
                ::freeaddrinfo(res);
                return s;
            }
            ::close(s);
            if (std::chrono::steady_clock::now() > until) {
                ::freeaddrinfo(res);
                throw WireError("cannot connect to " + host + ":" + std::to_string(port));
            }
            std::this_thread::sleep_for(std::chrono::milliseconds(100));
        }
    }

   public:
    // hosts[i] is host i's address; base_port as STARTMPC_BASE_PORT
    Endpoint(int rank, int count, int base_port, const std::vector<std::string>& hosts, int wait_s = 60)
        : rank_(rank), count_(count), fd_(count, -1) {
        if (count < 2 || rank < 0 || rank >= count || (int)hosts.size() != count)
            throw std::invalid_argument("bad party rank, count or host list");
        std::vector<std::thread> th;
        std::vector<std::string> err(count);
        for (int j = rank + 1; j < count; j++)
            th.emplace_back([&, j] {
                try {
                    fd_[j] = connect_to(hosts[j], base_port + count * rank + j, wait_s);
                } catch (const std::exception& e) {
                    err[j] = e.what();
                }
            });
        for (int i = 0; i < rank; i++)
            th.emplace_back([&, i] {
                try {
                    fd_[i] = listen_accept(base_port + count * i + rank);
                } catch (const std::exception& e) {
                    err[i] = e.what();
                }
            });
        for (auto& t : th) t.join();
        for (auto& e : err)
            if (!e.empty()) {
                close_all();
                throw WireError(e);
            }
    }

    // startmpc_init's environment, one worker thread
    static Endpoint from_env(int nparties, int wait_s = 60) {
        auto get = [](const char* k) -> const char* {
            const char* v = std::getenv(k);
            if (!v) throw std::invalid_argument(std::string(k) + " is not set");
            return v;
        };
        const int mode = std::atoi(get("STARTMPC_EXEC_MODE"));
        const int count = std::atoi(get("STARTMPC_HOST_COUNT"));
        const int rank = std::atoi(get("STARTMPC_HOST_RANK"));
        const int base = std::atoi(get("STARTMPC_BASE_PORT"));
        if (count != nparties) throw std::invalid_argument("STARTMPC_HOST_COUNT differs from the party count");
        std::vector<std::string> hosts;
        if (mode == 1) {
            std::stringstream ss(get("STARTMPC_HOST_LIST"));
            std::string h;
            while (std::getline(ss, h, ',')) hosts.push_back(h);
        } else {
            hosts.assign(count, "127.0.0.1");
        }
        return Endpoint(rank, count, base, hosts, wait_s);
    }

    Endpoint(Endpoint&& o) noexcept : rank_(o.rank_), count_(o.count_), fd_(std::move(o.fd_)) { o.fd_.clear(); }
    Endpoint(const Endpoint&) = delete;
    Endpoint& operator=(const Endpoint&) = delete;
    ~Endpoint() { close_all(); }
    void close_all() {
        for (int& f : fd_)
            if (f >= 0) {
                ::close(f);
                f = -1;
            }
    }

    int rank() const { return rank_; }
    int count() const { return count_; }
    // relative party id (as the reference's PartyID arguments) to absolute
    int abs(int rel) const { return ((rank_ + rel) % count_ + count_) % count_; }

    // sendShares: the vector's bytes, complete before return
    void send(int to, const void* p, size_t n) {
        const char* c = static_cast<const char*>(p);
        while (n) {
            const ssize_t k = ::send(fd_.at(to), c, n, MSG_NOSIGNAL);
            if (k <= 0) throw WireError("send to party " + std::to_string(to) + " failed");
            c += k;
            n -= (size_t)k;
        }
    }
    // receiveShares: exactly n bytes
    void recv(int from, void* p, size_t n) {
        char* c = static_cast<char*>(p);
        while (n) {
            const ssize_t k = ::recv(fd_.at(from), c, n, 0);
            if (k <= 0) throw WireError("party " + std::to_string(from) + " closed the connection");
            c += k;
            n -= (size_t)k;
        }
    }
    // exchangeShares: send to `to` while receiving from `from` (the reference
    // queues the send on its ring and receives meanwhile, so both directions
    // of a ring exchange proceed at once)
    void exchange(int to, const void* sp, int from, void* rp, size_t n) {
        std::string err;
        std::thread t([&] {
            try {
                send(to, sp, n);
            } catch (const std::exception& e) {
                err = e.what();
            }
        });
        try {
            recv(from, rp, n);
        } catch (...) {
            t.join();
            throw;
        }
        t.join();
        if (!err.empty()) throw WireError(err);
    }
};

}  // namespace nocopy
}  // namespace orq
