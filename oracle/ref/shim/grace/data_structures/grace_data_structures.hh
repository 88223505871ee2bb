#pragma once
#include <string>
#include <grace/data_structures/memory_defaults.hh>
#include <grace/data_structures/variable_properties.hh>
#include <grace/data_structures/variable_indices.hh>
