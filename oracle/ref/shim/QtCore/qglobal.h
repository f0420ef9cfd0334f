#pragma once
#define Q_DECL_EXPORT
#define Q_DECL_IMPORT
