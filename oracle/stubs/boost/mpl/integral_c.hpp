#include "ptstub_mpl.hpp"
