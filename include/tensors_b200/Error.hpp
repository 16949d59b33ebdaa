// tensors_b200::Sparse::Error and Check: C-ABI status codes as C++ exceptions,
// shared by the header-only mirrors (CholeskyDecomposition.hpp, MatrixCSR.hpp).
#pragma once

#include <stdexcept>
#include <string>

#include "../tensors_b200.h"

namespace tensors_b200 {
namespace Sparse {

class Error : public std::runtime_error
{
public:
    Error( int status, const std::string & what ) : std::runtime_error( what ), status_( status ) {}
    int Status() const noexcept { return status_; }
private:
    int status_;
};

inline int Check( int status )
{
    if( status < 0 ) { throw Error( status, tb_last_error() ); }
    return status;
}

} // namespace Sparse
} // namespace tensors_b200
