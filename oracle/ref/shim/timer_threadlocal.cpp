// Replacement of the reference's src/utils/timer.cpp for the thread-rank build.  TEST INFRASTRUCTURE ONLY.
// The reference keeps one process-wide TimerRegistry; with every rank a thread of one process that
// registry would be shared and raced.  Same interface (include/utils/timer.hpp), one registry per rank.
#include "timer.hpp"

#include <mpi.h>

#include <algorithm>
#include <iomanip>
#include <ostream>

namespace schwarz2lvl::utils {

TimerRegistry& TimerRegistry::instance()
{
    thread_local TimerRegistry reg;
    return reg;
}

void TimerRegistry::add(const std::string& name, double seconds)
{
    auto it = seconds_.find(name);
    if (it == seconds_.end()) {
        order_.push_back(name);
        seconds_[name] = seconds;
    } else {
        it->second += seconds;
    }
}

double TimerRegistry::get(const std::string& name) const
{
    auto it = seconds_.find(name);
    return it == seconds_.end() ? 0.0 : it->second;
}

void TimerRegistry::clear()
{
    order_.clear();
    seconds_.clear();
}

void TimerRegistry::report(MPI_Comm comm, std::ostream& os) const
{
    int rank = 0, size = 1;
    MPI_Comm_rank(comm, &rank);
    MPI_Comm_size(comm, &size);
    long long cnt = rank == 0 ? (long long)order_.size() : 0;
    MPI_Bcast(&cnt, 1, MPI_LONG_LONG, 0, comm);
    for (long long k = 0; k < cnt; ++k) {
        std::string name = rank == 0 ? order_[(size_t)k] : std::string();
        long long len = (long long)name.size();
        MPI_Bcast(&len, 1, MPI_LONG_LONG, 0, comm);
        name.resize((size_t)len);
        MPI_Bcast(name.data(), (int)len, MPI_CHAR, 0, comm);
        double v = get(name), mn = 0, mx = 0, sm = 0;
        MPI_Allreduce(&v, &mn, 1, MPI_DOUBLE, MPI_MIN, comm);
        MPI_Allreduce(&v, &mx, 1, MPI_DOUBLE, MPI_MAX, comm);
        MPI_Allreduce(&v, &sm, 1, MPI_DOUBLE, MPI_SUM, comm);
        if (rank == 0)
            os << "  " << std::left << std::setw(44) << name << std::right << std::fixed << std::setprecision(4) << mn
               << " " << sm / size << " " << mx << "\n";
    }
}

double TimerRegistry::maxOverRanks(MPI_Comm comm, const std::string& name) const
{
    double v = get(name), mx = 0;
    MPI_Allreduce(&v, &mx, 1, MPI_DOUBLE, MPI_MAX, comm);
    return mx;
}

ScopedTimer::ScopedTimer(std::string name) : name_(std::move(name)), start_(MPI_Wtime()) {}

ScopedTimer::~ScopedTimer() { TimerRegistry::instance().add(name_, MPI_Wtime() - start_); }

}  // namespace schwarz2lvl::utils
